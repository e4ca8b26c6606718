// Persistent engine: one cooperative launch runs all steps of a run for one group of instances.
//
// Instances are independent, so B is split into groups small enough that a group's neuron state
// (v, g f32 + refractory/flag byte = 9 B per instance-neuron, and its 4 B accumulator slice) fits
// in the shared memory of the whole GPU (148 x ~230 KB). Each CTA owns a contiguous slice of the group's (instance, neuron)
// pairs and keeps their state in shared memory for the whole run: per step, HBM/L2 traffic is
// only the synaptic-input accumulator slice (one TMA bulk load into shared memory, cleared behind
// it by bulk stores from a zero page), the CSR rows of the spikes that arrive next step, and the
// reductions they scatter.
//
// Epochs: the spikes of a step arrive n_delay steps later, so with K = (n_delay - 1) / 2 (at most
// MAX_EPOCH) the spikes of one epoch of K steps cannot arrive before the epoch after next. One grid
// barrier per epoch suffices: during an epoch the push warps scatter the work items that arrive in
// the next epoch into their accumulator slots (2K slots: tick mod 2K), while the neuron and
// listing warps step through the epoch with only a CTA-level barrier between steps.
//
// Warp roles of a CTA:
//   neuron warps (U, 26): per step, draw the next step's Poisson kicks into a shared bitmap while
//     the slice loads (issued at the end of the previous step when it lies in the same epoch),
//     then advance every owned pair;
//   listing warps (2): per step, list the previous step's spikes (counts, plastic rows, work items
//     of this CTA's segment of the group's list);
//   push warps (4): per epoch, scatter this CTA's share of the items arriving in the next epoch.
// Three bitmaps rotate: map[s%3] holds the kicks of step s, then (overwritten by the neuron warps)
// its spikes; map[(s+1)%3] receives the next kicks; the listing warps read and clear map[(s-1)%3].
// Every wait is bounded: after ~4 s a CTA raises the timeout flag and every CTA returns (the others
// read the flag in the grid barrier, so within an epoch a CTA waits only on its own bulk loads).
#pragma once
#include "engine.cuh"

namespace fb {

constexpr int PT = 1024;                // threads per CTA
constexpr int ZERO_PAGE = 4096;         // shared-memory zeros, the source of the clearing bulk stores
constexpr int LOAD_PIECE = 32768;       // bytes per bulk load of the accumulator slice
constexpr int SPK_BUF = 1024;           // spikes of one CTA and step listed in parallel
constexpr int IT_BUF = 384;             // work items of one CTA's epoch push staged in shared memory
constexpr int MAX_SPECIAL = 12;         // quads with a plastic target or a bias whose inputs are staged per step
constexpr long long BARRIER_TIMEOUT_CYCLES = 8000000000LL;   // ~4 s at 1.9 GHz
constexpr int MAX_EPOCH = 4;            // steps per epoch at most (accumulator slots: twice that; 8 slots of a
                                        // 16-instance group stay in L2, which measured faster than longer epochs)

constexpr int PUSH_WARPS = 4;                              // warps that scatter arriving items ...
constexpr int LIST_WARPS = 2;                              // ... that list the previous step's spikes ...
constexpr int PUSH_THREADS = 32 * PUSH_WARPS;
constexpr int LIST_THREADS = 32 * LIST_WARPS;
constexpr int U_THREADS = PT - PUSH_THREADS - LIST_THREADS;   // ... and the rest advance neurons

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
    const int2* ext_tab;      // per CTA: input pairs {k | instance << 18, ext slot}
    const int32_t* ext_off;   // (ctas + 1) offsets into ext_tab
    long long* trace;         // nullptr, or (steps, ctas, TRACE_SLOTS) clock64 stamps of each step's phases
    int64_t pushed_until;     // the arrivals of every tick < pushed_until are in the accumulators
    int32_t epoch;            // K: steps between grid barriers (2K accumulator slots, 2K + 1 <= n_delay)
    long long barrier_cycles; // the grid barrier's wait budget (SM clock cycles) before it times out
};

// Phase stamps (per step and CTA; SM clock cycles, compare within a CTA), in step order: 0 step
// start (the slice load issued right after), 4 the next step's kicks drawn, 1 ready to wait for the
// slice, 2 slice in shared memory, 3 neurons advanced; 8 listing warps done with the previous
// step; per epoch, at its first step: 7 push warps start, 10 push warps done; at its last step:
// 5 grid-barrier arrival, 6 grid-barrier exit (9 unused).
constexpr int TRACE_SLOTS = 11;

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


__device__ __forceinline__ void stamp(const PersistArgs& A, int32_t s, int slot)
{
    if (A.trace) A.trace[((int64_t)s * gridDim.x + blockIdx.x) * TRACE_SLOTS + slot] = clock64();
}

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
            if (clock64() - t0 > A.barrier_cycles) {
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

// Shared-memory layout of one CTA (bytes), for `per` pairs and accumulator type of `acc_bytes`.
struct PersistSmem {
    int64_t mbar, zero, acc, v, g, kbits, ref, misc, scan, pre, spk, ticks, items, special, kick, total, words_per_map;
    __host__ __device__ PersistSmem(int64_t per, int acc_bytes)
    {
        words_per_map = (per + 4 * PT) / 32 + 1;
        mbar = 0;
        zero = 128;
        acc = zero + ZERO_PAGE;
        v = acc + per * acc_bytes;
        g = v + per * 4;
        kbits = g + per * 4;                 // three bitmaps: the kicks of a step become its spikes
        ref = kbits + 3 * words_per_map * 4;
        misc = (ref + per + 15) / 16 * 16;   // 64 active flags, 16 counters
        scan = misc + 64 + 64;               // 32 block-scan partial sums
        pre = scan + 128;                    // MAX_EPOCH x MAX_SEG segment prefix entries
        spk = pre + 4 * MAX_EPOCH * MAX_SEG; // SPK_BUF spikes being listed
        ticks = spk + 4 * SPK_BUF;           // reset and stop ticks of up to 64 instances
        items = ticks + 2 * 64 * 8;          // IT_BUF staged work items of an epoch's push
        special = items + 16 * IT_BUF;      // MAX_SPECIAL quads: per step parity the accumulator values, plastic
                                            // deltas and kicks of their neurons; biases, posts, pair, instance
        kick = special + MAX_SPECIAL * (2 * 4 * (8 + 8 + 1) + 4 * 4 + 4 * 4 + 4 + 4);   // kick thresholds of
                                                                                       // 2 x U_THREADS inputs
        total = kick + 2 * U_THREADS * 4;
    }
};

__device__ __forceinline__ void u_sync() { asm volatile("bar.sync 1, %0;" ::"n"(U_THREADS) : "memory"); }
// barrier of the U threads that also ORs a predicate over them (so every U thread sees the same value)
__device__ __forceinline__ bool u_sync_or(bool pred)
{
    uint32_t out;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.or.pred p, 1, %2, p;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(out)
        : "r"((uint32_t)pred), "n"(U_THREADS)
        : "memory");
    return out != 0;
}
__device__ __forceinline__ void push_sync() { asm volatile("bar.sync 2, %0;" ::"n"(PUSH_THREADS) : "memory"); }
// step boundary between the neuron warps and the listing warps (the push warps run free in an epoch)
__device__ __forceinline__ void ul_sync() { asm volatile("bar.sync 4, %0;" ::"n"(U_THREADS + LIST_THREADS) : "memory"); }
__device__ __forceinline__ void list_sync() { asm volatile("bar.sync 3, %0;" ::"n"(LIST_THREADS) : "memory"); }

// bulk store shared -> global (16-byte aligned, size a multiple of 16), tracked by bulk groups
__device__ __forceinline__ void tma_store_1d(void* dst_gmem, const void* src_smem, uint32_t bytes)
{
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst_gmem), "r"(smem_u32(src_smem)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// A quad of the neuron loop with a plastic target or a biased neuron among its pairs, kept out of
// line so that the common loop body stays small. Advances pairs 0..nvalid-1 of the quad in
// shared memory (xs, vs, gs, fs) and returns their spike bits. Plastic input arriving at a target
// is read from pring_row[ppost_of_i[j]] and cleared (L2 only: other SMs pushed it); a biased
// pair's bias is bias_row[ext_idx_i[j]]. The global loads of the four pairs are issued together
// (indices, then values), so a quad waits for two round trips to L2, not eight.
template <typename AccT, int PLASTIC>
__device__ __noinline__ uint32_t quad_special(const AccT* xs, float* vs, float* gs, uint8_t* fs, uint32_t kick4,
                                              int nvalid, int64_t* pring_row, const int32_t* ppost_of_i,
                                              const float* bias_row, const int32_t* ext_idx_i, const Lif<float> L,
                                              int n_ref)
{
    uint32_t f[4];
    int32_t pp[4], ei[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        f[j] = j < nvalid ? (uint32_t)fs[j] : 0u;
        pp[j] = (PLASTIC && (f[j] & 0x40)) ? __ldg(ppost_of_i + j) : -1;
        ei[j] = (f[j] & 0x80) ? __ldg(ext_idx_i + j) : -1;
    }
    int64_t px[4];
    float bias[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        px[j] = pp[j] >= 0 ? (int64_t)__ldcg(reinterpret_cast<const long long*>(pring_row + pp[j])) : 0;
        bias[j] = ei[j] >= 0 ? bias_row[ei[j]] : 0.0f;
    }
    uint32_t spk4 = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        if (j >= nvalid) continue;
        float buf = acc_to_real<float>(xs[j], L.w_syn);
        if (pp[j] >= 0) buf = add_rn(buf, from_q32<float>(px[j]));
        int r = (int)(f[j] & 0x3f);
        const bool hb = (f[j] & 0x80) != 0;
        float v = vs[j], g = gs[j];
        if (lif_step<float>(v, g, r, buf, hb, bias[j], (kick4 >> j) & 1u, L, n_ref, true)) spk4 |= 1u << j;
        vs[j] = v;
        gs[j] = g;
        fs[j] = (uint8_t)((f[j] & 0xc0) | (uint32_t)r);
    }
#pragma unroll
    for (int j = 0; j < 4; j++)
        if (pp[j] >= 0 && px[j] != 0) pring_row[pp[j]] = 0;
    return spk4;
}

__device__ __forceinline__ void load4(const int32_t* p, int32_t (&x)[4])
{
    const int4 v = *reinterpret_cast<const int4*>(p);
    x[0] = v.x; x[1] = v.y; x[2] = v.z; x[3] = v.w;
}
__device__ __forceinline__ void load4(const int64_t* p, int64_t (&x)[4])
{
    const longlong2 a = reinterpret_cast<const longlong2*>(p)[0], b = reinterpret_cast<const longlong2*>(p)[1];
    x[0] = a.x; x[1] = a.y; x[2] = b.x; x[3] = b.y;
}

// Poisson kicks of step s (tick t) for this CTA's input pairs, OR-ed into `map` (threads tid0, stride).
// Entries are taken four at a time so that their loads are in flight together.
template <bool RASTER>
__device__ __forceinline__ void kicks_into(const DevNet& N, const DevState& S, const PersistArgs& A, uint32_t* map,
                                           int32_t s, int64_t t, uint32_t step_no, int32_t b0, int32_t G, int64_t lo,
                                           int32_t e0, int32_t e1, int tid0, int stride, const int64_t* stop)
{
    const int32_t n = (int32_t)N.n, np = (int32_t)N.n_pad;
    constexpr int BATCH = 4;
    for (int32_t e = e0 + tid0; e < e1; e += BATCH * stride) {
        int2 en[BATCH];
#pragma unroll
        for (int u = 0; u < BATCH; u++) en[u] = (e + u * stride < e1) ? __ldg(A.ext_tab + e + u * stride) : make_int2(0, -1);
        bool hit[BATCH];
#pragma unroll
        for (int u = 0; u < BATCH; u++) {
            const int32_t k = en[u].x & 0x3ffff, bl = en[u].x >> 18;
            hit[u] = false;
            if (en[u].y < 0 || bl >= G || t >= stop[bl]) continue;
            const int32_t b = b0 + bl;
            const int32_t i = (int32_t)(lo + k - (int64_t)bl * np);
            hit[u] = kick_of<RASTER>(S, A.kicks, A.words, N.B, s, b, en[u].y, (uint32_t)((int64_t)b * n + i), step_no);
        }
#pragma unroll
        for (int u = 0; u < BATCH; u++)
            if (hit[u]) atomicOr(map + ((en[u].x & 0x3ffff) >> 5), 1u << (en[u].x & 31));
    }
}

// Kick threshold of an input of probability p: with u = h >> 8 < 2^24 the draw u * 2^-24 < p of
// hash_kick holds exactly when u < ceil(p * 2^24) (the product is exact in float); 0 for p <= 0.
__device__ __forceinline__ int32_t kick_threshold(float p)
{
    return p > 0.0f ? (int32_t)fminf(ceilf(__fmul_rn(p, 16777216.0f)), 16777217.0f) : 0;
}

// The Poisson kicks of a U thread's first two input pairs, held for the launch (the probabilities
// are constant during a launch): the pair and instance {local pair | instance << 18} in registers,
// the thresholds in shared memory; one hash per pair and step.
__device__ __forceinline__ void kicks_held(const DevNet& N, const DevState& S, const int32_t (&kx)[2], const int32_t* s_kt,
                                           int tid, uint32_t* map, int64_t t, uint32_t step_no, int32_t b0, int64_t lo,
                                           const int64_t* stop)
{
    const uint32_t sm = step_no * 0x9e3779b9u;
#pragma unroll
    for (int u = 0; u < 2; u++) {
        const int32_t thr = s_kt[u * U_THREADS + tid];
        if (thr <= 0) continue;
        const int32_t k = kx[u] & 0x3ffff, bl = kx[u] >> 18;
        if (t >= stop[bl]) continue;
        const int32_t b = b0 + bl;
        const int32_t i = (int32_t)(lo + k - (int64_t)bl * N.n_pad);
        const uint32_t h = mix32((uint32_t)((int64_t)b * N.n + i) ^ mix32(sm ^ mix32(S.seed + (uint32_t)b)));
        if ((int32_t)(h >> 8) < thr) atomicOr(map + (k >> 5), 1u << (k & 31));
    }
}

// Exclusive prefix of `x` over the threads tid0 = 0..stride-1 (whole warps) and the total; uses
// `scratch` (stride / 32 entries of shared memory) and two `sync`s.
template <typename Sync>
__device__ __forceinline__ int block_scan(int x, int* total, int32_t* scratch, int tid0, int stride, Sync sync)
{
    const int lane = tid0 & 31, warp = tid0 >> 5;
    int incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) scratch[warp] = incl;
    sync();
    int before = 0, all = 0;
    for (int w = 0; w < stride / 32; w++) {
        const int v = scratch[w];
        before += w < warp ? v : 0;
        all += v;
    }
    sync();
    *total = all;
    return before + incl - x;
}

// One spike of the listing: pair k of this CTA fired at step s (tick t). Counts it, pushes its
// plastic row, records it, and appends its work items to this CTA's list segment (cursor s_cnt[1]).
template <int PLASTIC, bool RECORD>
__device__ __forceinline__ void list_one(const DevNet& N, const DevState& S, const PersistArgs& A, int2* list, int32_t k,
                                         int32_t s, int64_t t, int32_t b0, int64_t lo, int32_t* s_cnt)
{
    const int32_t np = (int32_t)N.n_pad;
    const int64_t lp = lo + k;
    const int32_t bl = (int32_t)(lp / np), i = (int32_t)(lp - (int64_t)bl * np);
    const int32_t b = b0 + bl;
    red_add(A.counts + (int64_t)b * N.n + i, 1);
    const int nch = (int)((__ldg(N.rowptr + i + 1) - __ldg(N.rowptr + i) + CHUNK - 1) / CHUNK);
    if (PLASTIC == 2) push_plastic_row_batched(N, S, t, b, i);
    else if (PLASTIC) push_plastic_row(N, S, t, b, i);
    if (RECORD) {
        if (A.step_counts) atomicAdd(A.step_counts + (int64_t)s * N.B + b, 1);
        if (A.step_digest)
            atomicAdd(reinterpret_cast<unsigned long long*>(A.step_digest + (int64_t)s * N.B + b),
                      (unsigned long long)spike_tag((uint64_t)i));
    }
    if (nch == 0) return;
    int base = atomicAdd(&s_cnt[1], nch);
    for (int c = 0; c < nch; c++, base++) {
        if (base < S.cap_c) list[base] = make_item(N, i, b, c);
        else atomicExch(S.err, 1);
    }
}

// The spikes of step s (tick t) recorded in `map`: counts, plastic rows, records, and the work items
// of this CTA's segment of the group's list; the segment's count is stored at the end. Clears `map`.
// The spikes are first gathered into `spk` (SPK_BUF entries) so that each is then handled by its
// own thread, their memory accesses all in flight at once; spikes beyond the buffer are handled
// where they are found. Threads tid0 = 0..stride-1 (whole warps) all call it (synchronised by `sync`).
template <int PLASTIC, bool RECORD, typename Sync>
__device__ __forceinline__ void list_spikes(const DevNet& N, const DevState& S, const PersistArgs& A, uint32_t* map,
                                            int32_t s, int64_t t, int32_t b0, int32_t q, int64_t lo, int32_t used_words,
                                            int32_t* s_cnt, int32_t* scratch, int32_t* spk, int tid0, int stride,
                                            Sync sync)
{
    const int64_t slot = pos_mod(t, N.R);
    int2* list = list_of(S, slot, q, blockIdx.x);
    const int32_t wpt = (used_words + stride - 1) / stride;      // contiguous words per thread
    const int32_t wa = min(tid0 * wpt, used_words), wb = min(wa + wpt, used_words);
    int mine = 0;
    for (int32_t w = wa; w < wb; w++) mine += __popc(map[w]);
    int total = 0;
    int pos = block_scan(mine, &total, scratch, tid0, stride, sync);
    if (mine) {
        for (int32_t w = wa; w < wb; w++) {
            uint32_t m = map[w];
            if (!m) continue;
            map[w] = 0u;
            for (; m; m &= m - 1, pos++) {
                const int32_t k = w * 32 + __ffs(m) - 1;
                if (pos < SPK_BUF) spk[pos] = k;
                else list_one<PLASTIC, RECORD>(N, S, A, list, k, s, t, b0, lo, s_cnt);
            }
        }
    }
    sync();
    for (int j = tid0; j < min(total, SPK_BUF); j += stride)
        list_one<PLASTIC, RECORD>(N, S, A, list, spk[j], s, t, b0, lo, s_cnt);
    sync();
    if (tid0 == 0) {
        *count_of(S, slot, q, blockIdx.x) = s_cnt[1];
        s_cnt[1] = 0;
    }
}

// Bulk load of this CTA's accumulator slice (`bytes` from global `src`) into shared memory,
// completing on `mbar` (one transaction per step: the waits alternate parity).
template <typename AccT>
__device__ __forceinline__ void issue_slice(const AccT* src, AccT* sacc, uint32_t bytes, uint64_t* mbar)
{
    fence_proxy_async_global();
    mbar_expect_tx(mbar, bytes);
    for (uint32_t off = 0; off < bytes; off += LOAD_PIECE)
        tma_load_1d(reinterpret_cast<uint8_t*>(sacc) + off, reinterpret_cast<const uint8_t*>(src) + off,
                    min((uint32_t)LOAD_PIECE, bytes - off), mbar);
}

// Push warps: scatter this CTA's share of the work items that arrive at ticks [a0, a1) into their
// accumulator slots, one arrival tick after the other (its list is the spikes of tick a - n_delay).
template <typename AccT, int LANES>
__device__ __forceinline__ void push_arrivals(const DevNet& N, const DevState& S, int32_t q, int32_t b0, int64_t a0,
                                              int64_t a1, int32_t* s_pre, int32_t* s_cnt, const int64_t* s_reset,
                                              const int64_t* s_stop, int ptid)
{
    for (int64_t a = a0; a < a1; a++) {
        const int64_t sp = a - N.n_delay;
        if (sp < 0) continue;
        const int par = (int)(a & 1);
        int32_t* pre = s_pre + par * MAX_SEG;
        if (ptid < 32) {
            const int32_t tot = segment_prefix(S, pos_mod(sp, N.R), q, pre);
            if (ptid == 0) s_cnt[2 + par] = tot;
        }
        push_sync();
        const int64_t total = s_cnt[2 + par];   // this CTA's share: a contiguous range of items
        const int64_t g0 = total * blockIdx.x / gridDim.x, g1 = total * (blockIdx.x + 1) / gridDim.x;
        push_range<AccT, LANES>(N, S, a - 1, q, acc_slot<AccT>(N, S, a), pre, g0, g1, ptid / LANES,
                                PUSH_THREADS / LANES, ptid % LANES, s_reset, s_stop, b0);
    }
}

// Push warps, one epoch: this CTA's shares of the lists arriving at ticks [a0, a1) (at most
// MAX_EPOCH lists) scattered with every memory access of a phase in flight at once:
//   1. the segment prefixes of all lists (each warp takes whole lists);
//   2. every item of the shares loaded once (thread j takes a contiguous run), filtered by the
//      instance ticks, recorded in shared memory as {first entry, entries, instance, arrival}, and
//      numbered by 8-entry groups (a scan over the push threads);
//   3. the groups spread over all push threads, two in flight per thread.
// Items beyond IT_BUF follow list by list (push_range).
template <typename AccT, int LANES>
__device__ __forceinline__ void push_epoch(const DevNet& N, const DevState& S, int32_t q, int32_t b0, int64_t a0,
                                           int64_t a1, int32_t* s_pre, int32_t* s_cnt, int32_t* scratch, int4* recs,
                                           const int64_t* s_reset, const int64_t* s_stop, int ptid)
{
    const int nl = (int)(a1 - a0);
    const int warp = ptid >> 5;
    for (int k = warp; k < nl; k += PUSH_WARPS) {
        const int64_t sp = a0 + k - N.n_delay;
        int32_t tot = 0;
        if (sp >= 0) tot = segment_prefix(S, pos_mod(sp, N.R), q, s_pre + k * MAX_SEG);
        if ((ptid & 31) == 0) s_cnt[8 + k] = sp >= 0 ? tot : 0;       // list totals: s_cnt[8 .. 8+MAX_EPOCH)
    }
    push_sync();
    // shares and their flattened offsets (every thread computes the same small table)
    int64_t g0[MAX_EPOCH], off[MAX_EPOCH + 1];
    off[0] = 0;
#pragma unroll
    for (int k = 0; k < MAX_EPOCH; k++) {
        const int64_t total = k < nl ? s_cnt[8 + k] : 0;
        g0[k] = total * blockIdx.x / gridDim.x;
        off[k + 1] = off[k] + (total * (blockIdx.x + 1) / gridDim.x - g0[k]);
    }
    const int64_t M = off[MAX_EPOCH];
    const int32_t m = (int32_t)min(M, (int64_t)IT_BUF);
    // 2. stage the items: thread ptid takes records [ptid * c, (ptid + 1) * c)
    const int32_t c = (m + PUSH_THREADS - 1) / PUSH_THREADS;
    const int32_t r0 = min(ptid * c, m), r1 = min(r0 + c, m);
    int groups = 0;
    for (int32_t j = r0; j < r1; j++) {
        int k = 0;
        while (k + 1 < MAX_EPOCH && off[k + 1] <= j) k++;
        const int64_t g = g0[k] + (j - off[k]);
        const int32_t* pre = s_pre + k * MAX_SEG;
        int32_t lo = 0, hi = S.n_seg - 1;                        // first segment whose prefix exceeds g
        while (lo < hi) {
            const int32_t mid = (lo + hi) >> 1;
            if (pre[mid] > g) hi = mid;
            else lo = mid + 1;
        }
        const int64_t sp = a0 + k - N.n_delay;
        const int2 item = __ldcg(list_of(S, pos_mod(sp, N.R), q, lo) + (g - (lo > 0 ? pre[lo - 1] : 0)));
        const int32_t bl = (item.y >> CHUNK_BITS) - b0;
        int32_t len = item.y & ((1 << CHUNK_BITS) - 1);
        if (sp < s_reset[bl] || a0 + k >= s_stop[bl]) len = 0;
        recs[j] = make_int4(item.x, len, bl | (k << 8), 0);
        groups += (len + 7) / 8;
    }
    int all = 0;
    int base = block_scan(groups, &all, scratch, ptid, PUSH_THREADS, []() { push_sync(); });
    for (int32_t j = r0; j < r1; j++) {
        recs[j].w = base;
        base += (recs[j].y + 7) / 8;
    }
    push_sync();
    // 3. the 8-entry groups, two in flight per thread
    const int64_t np = N.n_pad;
    const int64_t slot_stride = (int64_t)N.B * np;
    AccT* acc0 = reinterpret_cast<AccT*>(S.acc);
    auto locate = [&](int32_t gi) {                              // last record whose first group <= gi
        int32_t lo = 0, hi = m - 1;
        while (lo < hi) {
            const int32_t mid = (lo + hi + 1) >> 1;
            if (recs[mid].w <= gi) lo = mid;
            else hi = mid - 1;
        }
        return recs[lo];
    };
    auto target = [&](const int4& r) {
        const int k = r.z >> 8, bl = r.z & 0xff;
        return acc0 + pos_mod(a0 + k, S.n_slots) * slot_stride + (int64_t)(b0 + bl) * np;
    };
    for (int32_t ga = ptid; ga < all; ga += 2 * PUSH_THREADS) {
        const int32_t gb = ga + PUSH_THREADS;
        const int4 ra = locate(ga);
        Edges8<AccT> ea, eb;
        ea.load(N, (int64_t)(uint32_t)ra.x + 8 * (int64_t)(ga - ra.w));
        int4 rb = ra;
        if (gb < all) {
            rb = locate(gb);
            eb.load(N, (int64_t)(uint32_t)rb.x + 8 * (int64_t)(gb - rb.w));
        }
        AccT* ta = target(ra);
#pragma unroll
        for (int u = 0; u < 8; u++)
            if (ea.w[u] != 0) red_add(ta + ea.c[u], ea.w[u]);
        if (gb < all) {
            AccT* tb = target(rb);
#pragma unroll
            for (int u = 0; u < 8; u++)
                if (eb.w[u] != 0) red_add(tb + eb.c[u], eb.w[u]);
        }
    }
    // items beyond the stage, list by list
    if (M > IT_BUF) {
        for (int k = 0; k < nl; k++) {
            const int64_t lo_j = max(off[k], (int64_t)IT_BUF), hi_j = off[k + 1];
            if (lo_j >= hi_j) continue;
            push_range<AccT, LANES>(N, S, a0 + k - 1, q, acc_slot<AccT>(N, S, a0 + k), s_pre + k * MAX_SEG,
                                    g0[k] + (lo_j - off[k]), g0[k] + (hi_j - off[k]), ptid / LANES,
                                    PUSH_THREADS / LANES, ptid % LANES, s_reset, s_stop, b0);
        }
    }
    push_sync();                                 // the records are free again
}

// One launch runs `A.steps` steps of the instances [b0, b0 + G) (group q); the warp roles and the
// bitmap rotation are described at the top of this file.
template <typename AccT, bool RASTER, int PLASTIC, bool RECORD, int LANES>
__global__ void __launch_bounds__(PT, 1)
    k_persist(const DevNet N, const DevState S, const PersistArgs A, int32_t b0, int32_t G, int32_t q, int64_t per)
{
    extern __shared__ __align__(128) uint8_t smem[];
    const PersistSmem lay(per, (int)sizeof(AccT));
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + lay.mbar);
    const uint8_t* zero = smem + lay.zero;
    AccT* sacc = reinterpret_cast<AccT*>(smem + lay.acc);
    float* sv = reinterpret_cast<float*>(smem + lay.v);
    float* sg = reinterpret_cast<float*>(smem + lay.g);
    uint32_t* maps = reinterpret_cast<uint32_t*>(smem + lay.kbits);
    uint8_t* sr = smem + lay.ref;            // bits 0-5 refractory, 6 plastic target, 7 nonzero bias
    uint8_t* s_active = smem + lay.misc;
    int32_t* s_cnt = reinterpret_cast<int32_t*>(smem + lay.misc + 64);   // -, list cursor, push totals
    int32_t* s_scan = reinterpret_cast<int32_t*>(smem + lay.scan);
    int32_t* s_pre = reinterpret_cast<int32_t*>(smem + lay.pre);         // segment prefixes x2 (step parity)
    int32_t* s_spk = reinterpret_cast<int32_t*>(smem + lay.spk);
    int64_t* s_reset = reinterpret_cast<int64_t*>(smem + lay.ticks);     // per instance of the group
    int64_t* s_stop = s_reset + 64;
    int4* s_items = reinterpret_cast<int4*>(smem + lay.items);
    int64_t* s_sp_acc = reinterpret_cast<int64_t*>(smem + lay.special);        // [parity][neuron] accumulator
    int64_t* s_sp_pl = s_sp_acc + 2 * 4 * MAX_SPECIAL;                         // [parity][neuron] plastic delta
    float* s_sp_bias = reinterpret_cast<float*>(s_sp_pl + 2 * 4 * MAX_SPECIAL); // biases (x4)
    int32_t* s_sp_pp = reinterpret_cast<int32_t*>(s_sp_bias + 4 * MAX_SPECIAL); // plastic post index or -1 (x4)
    int32_t* s_sp_k = s_sp_pp + 4 * MAX_SPECIAL;                               // local pair of the quad
    int32_t* s_sp_bl = s_sp_k + MAX_SPECIAL;                                   // its instance in the group
    uint8_t* s_sp_kick = reinterpret_cast<uint8_t*>(s_sp_bl + MAX_SPECIAL);    // [parity][neuron] kick bit
    const Lif<float> L = N.L32;
    const int n_ref = N.n_ref;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int32_t n = (int32_t)N.n, np = (int32_t)N.n_pad;
    const int64_t lo = (int64_t)blockIdx.x * per;
    const int32_t cnt = (int32_t)max((int64_t)0, min(per, (int64_t)G * np - lo));
    const int64_t acc_base = (int64_t)b0 * np + lo;       // accumulator index of local pair 0
    float* V = reinterpret_cast<float*>(S.v);
    float* Gs = reinterpret_cast<float*>(S.g);
    const int32_t e0 = A.ext_off[blockIdx.x], e1 = A.ext_off[blockIdx.x + 1];
    const int32_t wpm = (int32_t)lay.words_per_map;
    const int32_t used_words = (cnt + 31) / 32;

    // ---- load this CTA's state into shared memory ------------------------------------------
    for (int32_t k = tid; k < cnt; k += PT) {
        const int64_t lp = lo + k;
        const int32_t bl = (int32_t)(lp / np), i = (int32_t)(lp - (int64_t)bl * np);
        uint8_t f = 0;
        if (i < n) {
            const int64_t gp = (int64_t)(b0 + bl) * n + i;
            sv[k] = V[gp];
            sg[k] = Gs[gp];
            f = (uint8_t)S.ref[gp];
            if (PLASTIC && N.ppost_of[i] >= 0) f |= 0x40;
        }
        sr[k] = f;
    }
    for (int32_t w = tid; w < 3 * wpm; w += PT) maps[w] = 0u;
    for (int32_t z = tid; z < ZERO_PAGE / 4; z += PT) reinterpret_cast<uint32_t*>(smem + lay.zero)[z] = 0u;
    fence_proxy_async_shared();                                  // zero page visible to bulk copies
    if (tid == 0) {
        mbar_init(mbar, 1);
        fence_mbar_init();
        for (int c = 0; c < 16; c++) s_cnt[c] = 0;
    }
    if (tid < G) {                                               // the ticks stay constant during a launch
        s_reset[tid] = S.reset_tick[b0 + tid];
        s_stop[tid] = S.stop_tick[b0 + tid];
    }
    __syncthreads();
    for (int32_t e = e0 + tid; e < e1; e += PT) {               // bias is constant during a launch
        const int2 en = __ldg(A.ext_tab + e);
        const int32_t k = en.x & 0x3ffff, bl = en.x >> 18;
        if (bl < G && S.bias_ext[(int64_t)(b0 + bl) * S.n_ext + en.y] != 0.0f) sr[k] |= 0x80;
    }
    __syncthreads();
    // the quads with a plastic target or a biased neuron (constant during a launch), listed with their
    // posts and biases: the neuron loop skips them; the neuron warps stage each step's inputs of their
    // neurons (accumulator value, kick, plastic delta) and the listing warps advance them one per
    // thread at the start of the next step, before they list that step's spikes: the out-of-line
    // call and its local-memory traffic leave the neuron warps' path
    for (int32_t k = 4 * tid; k < cnt; k += 4 * PT) {
        const uint32_t fl = *reinterpret_cast<const uint32_t*>(sr + k);
        if ((fl & 0xc0c0c0c0u) == 0) continue;
        const int e = atomicAdd(&s_cnt[12], 1);
        if (e >= MAX_SPECIAL) continue;
        const int64_t lp = lo + k;
        const int32_t bl = (int32_t)(lp / np), i = (int32_t)(lp - (int64_t)bl * np);
        s_sp_k[e] = k;
        s_sp_bl[e] = bl;
        for (int j = 0; j < 4; j++) {
            const uint32_t f = (fl >> (8 * j)) & 0xffu;
            const bool in = i + j < n;
            s_sp_pp[4 * e + j] = (PLASTIC && in && (f & 0x40)) ? N.ppost_of[i + j] : -1;
            s_sp_bias[4 * e + j] = (in && (f & 0x80)) ? S.bias_ext[(int64_t)(b0 + bl) * S.n_ext + S.ext_idx[i + j]] : 0.0f;
        }
    }
    // a U thread's first two input pairs with their kick thresholds (the rest, if a CTA has more
    // than 2 x U_THREADS, are drawn from the table every step)
    int32_t kx[2] = {0, 0};
    int32_t* s_kt = reinterpret_cast<int32_t*>(smem + lay.kick);
    if (!RASTER && tid < U_THREADS) {
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const int32_t ee = e0 + tid + u * U_THREADS;
            int32_t thr = 0;
            if (ee < e1) {
                const int2 en = __ldg(A.ext_tab + ee);
                const int32_t bl = en.x >> 18;
                if (en.y >= 0 && bl < G) {
                    kx[u] = en.x;
                    thr = kick_threshold(S.p_ext[(int64_t)(b0 + bl) * S.n_ext + en.y]);
                }
            }
            s_kt[u * U_THREADS + tid] = thr;
        }
    }
    if (A.steps > 0) kicks_into<RASTER>(N, S, A, maps, 0, A.t0, A.step0, b0, G, lo, e0, e1, tid, PT, s_stop);
    __syncthreads();

    unsigned int barriers = 0;
    const bool all_staged = s_cnt[12] <= MAX_SPECIAL;
    // staged special quads of this CTA (none when it has more than MAX_SPECIAL: then all of them take
    // the out-of-line call inside the neuron loop)
    const int n_sp = all_staged ? s_cnt[12] : 0;
    // a staged neuron e of step s_prev (tick t_prev) from its staged inputs; its spike bit into that
    // step's bitmap (before the step is listed)
    auto advance_staged = [&](int32_t s_prev, int64_t t_prev, int e) {
        const int sp = e >> 2, j = e & 3, par = s_prev & 1;
        const int32_t kq = s_sp_k[sp], blq = s_sp_bl[sp];
        const int32_t iq = (int32_t)(lo + kq - (int64_t)blq * np) + j;
        if (iq >= n || t_prev >= s_stop[blq]) return;
        const int32_t kk = kq + j;
        const uint32_t f = sr[kk];
        float buf = acc_to_real<float>((AccT)s_sp_acc[par * 4 * MAX_SPECIAL + e], L.w_syn);
        if (PLASTIC && (f & 0x40)) buf = add_rn(buf, from_q32<float>(s_sp_pl[par * 4 * MAX_SPECIAL + e]));
        int r = (int)(f & 0x3f);
        float v = sv[kk], g = sg[kk];
        const bool hit = lif_step<float>(v, g, r, buf, (f & 0x80) != 0, s_sp_bias[4 * sp + j],
                                         s_sp_kick[par * 4 * MAX_SPECIAL + e], L, n_ref, true);
        sv[kk] = v;
        sg[kk] = g;
        sr[kk] = (uint8_t)((f & 0xc0) | (uint32_t)r);
        if (hit) atomicOr(maps + (s_prev % 3) * wpm + (kk >> 5), 1u << (kk & 31));
    };
    int32_t* err = S.err;
    const uint32_t acc_bytes = (uint32_t)cnt * (uint32_t)sizeof(AccT);
    const int32_t i0 = (int32_t)((lo + 4 * tid) % np), bl0 = (int32_t)((lo + 4 * tid) / np);
    const int K = A.epoch;
    const int64_t t_end = A.t0 + A.steps;
    const bool is_u = tid < U_THREADS, is_p = !is_u && tid < U_THREADS + PUSH_THREADS;
    const int ptid = tid - U_THREADS, lt = tid - U_THREADS - PUSH_THREADS;
    int64_t pushed = A.pushed_until;                            // the arrivals of ticks < pushed are complete
    int32_t last = -1;                                          // step whose spikes still need listing
    bool stop = false;
    bool staged = false;                                        // this step's slice load was issued early

    // ---- prologue: the arrivals of the first epoch not in the accumulators yet -----------------
    if (A.steps > 0) {
        const int64_t a1 = min(A.t0 + K, t_end + 1);
        if (pushed < a1) {
            if (is_p) push_arrivals<AccT, LANES>(N, S, q, b0, pushed, a1, s_pre, s_cnt, s_reset, s_stop, ptid);
            barriers++;
            stop = grid_barrier(A, barriers * gridDim.x, err, 1);
            pushed = a1;
        }
    }
    // ---- epochs of K steps, one grid barrier each ---------------------------------------------
    for (int32_t ep0 = 0; ep0 < A.steps && !stop; ep0 += K) {
        const int32_t ep1 = min(ep0 + K, A.steps);
        const int64_t te_end = A.t0 + ep1;
        // pushes of this epoch: the arrivals of the next epoch (and of the tick after the run)
        const int64_t pa0 = max(pushed, te_end), pa1 = min(te_end + K, t_end + 1);
        if (is_p) {
            if (ptid == 0) stamp(A, ep0, 7);
            if (pa0 < pa1)
                push_epoch<AccT, LANES>(N, S, q, b0, pa0, pa1, s_pre, s_cnt, s_scan + 16, s_items, s_reset, s_stop,
                                        ptid);
            if (ptid == 0) stamp(A, ep0, 10);
        } else {
            for (int32_t s = ep0; s < ep1; s++) {
                const int64_t t = A.t0 + s;
                const uint32_t step_no = A.step0 + (uint32_t)s;
                const AccT* acc = acc_slot<AccT>(N, S, t);
                uint32_t* map = maps + (s % 3) * wpm;
                ul_sync();                       // neuron and listing warps: step boundary
                if (is_u) {
                    if (tid == 0) stamp(A, s, 0);
                    if (tid == 0 && cnt > 0 && !staged)
                        issue_slice(acc + acc_base, sacc, acc_bytes, mbar);
                    if (tid < G) s_active[tid] = t < s_stop[tid];
                    // a staged neuron's thread: its kick of this step (the loop below overwrites the
                    // word) and its plastic delta of this tick (complete since the last grid barrier),
                    // whose load is stored for the listing warps only after the loop
                    int64_t sp_pl = 0;
                    int64_t* sp_pl_at = nullptr;
                    if (tid < 4 * n_sp) {
                        const int sp = tid >> 2, j = tid & 3, blq = s_sp_bl[sp], kk = s_sp_k[sp] + j;
                        s_sp_kick[(s & 1) * 4 * MAX_SPECIAL + tid] = (uint8_t)((map[kk >> 5] >> (kk & 31)) & 1u);
                        const int32_t pp = s_sp_pp[4 * sp + j];
                        if (PLASTIC && pp >= 0 && t < s_stop[blq]) {
                            sp_pl_at = S.pring + (pos_mod(t, N.R_pl) * N.B + (b0 + blq)) * (int64_t)N.n_ppost + pp;
                            sp_pl = (int64_t)__ldcg(reinterpret_cast<const long long*>(sp_pl_at));
                        }
                    }
                    // ---- the next step's kicks, in the shadow of the slice load: they depend on nothing
                    //      this step computes, and their bitmap was listed and cleared in the last step
                    if (s + 1 < A.steps) {
                        uint32_t* mnext = maps + ((s + 1) % 3) * wpm;
                        if (RASTER) {
                            kicks_into<RASTER>(N, S, A, mnext, s + 1, t + 1, step_no + 1u, b0, G, lo, e0, e1, tid, U_THREADS,
                                               s_stop);
                        } else {
                            kicks_held(N, S, kx, s_kt, tid, mnext, t + 1, step_no + 1u, b0, lo, s_stop);
                            if (e1 - e0 > 2 * U_THREADS)
                                kicks_into<RASTER>(N, S, A, mnext, s + 1, t + 1, step_no + 1u, b0, G, lo, e0 + 2 * U_THREADS,
                                                   e1, tid, U_THREADS, s_stop);
                        }
                    }
                    if (tid == 0) stamp(A, s, 4);
                    // this CTA's list segment consumed by the pushes for tick t starts empty (the
                    // step engine appends to it)
                    if (tid == 64) *count_of(S, pos_mod(t - N.n_delay, N.R), q, blockIdx.x) = 0;
                    if (tid == 0) stamp(A, s, 1);
                    bool ok = true;
                    if (cnt > 0 && tid == 0)
                        ok = stage_wait(mbar, (uint32_t)(s & 1), A, err, s + 1);
                    ok = !u_sync_or(!ok);        // one thread waited; every U thread agrees on the outcome
                    if (cnt > 0 && ok) (void)mbar_try_wait(mbar, (uint32_t)(s & 1));   // completed: acquire only
                    if (tid == 0) stamp(A, s, 2);
                    if (cnt > 0 && ok && tid < 32) {     // the slice is in shared memory: clear it in global
                        AccT* accw = const_cast<AccT*>(acc) + acc_base;   // memory, a zero page per lane of warp 0
                        bool any = false;
                        for (uint32_t off = (uint32_t)tid * ZERO_PAGE; off < acc_bytes; off += 32u * ZERO_PAGE) {
                            tma_store_1d(reinterpret_cast<uint8_t*>(accw) + off, zero, min((uint32_t)ZERO_PAGE, acc_bytes - off));
                            any = true;
                        }
                        if (any) bulk_commit();
                    }
                // ---- advance every owned pair, four consecutive pairs per thread (a quad never straddles
                //      two instances: rows are padded to 16); the step's kicks are read from the map and
                //      its spikes written back into it --------------------------------------------------
                if (ok && tid < 4 * n_sp)             // the staged neurons' accumulator values of this step
                    s_sp_acc[(s & 1) * 4 * MAX_SPECIAL + tid] = (int64_t)sacc[s_sp_k[tid >> 2] + (tid & 3)];
                if (ok) {
                    int32_t i = i0, bl = bl0;
                    bool act = bl < 64 && s_active[bl];         // this instance still runs (read once per row)
                    const int sh = 4 * (lane & 7);              // this quad's nibble in its 32-bit word
                    for (int32_t kb = 0; kb < cnt; kb += 4 * U_THREADS) {
                        const int32_t k = kb + 4 * tid;
                        const uint32_t kick4 = (map[k >> 5] >> sh) & 15u;
                        uint32_t spk4 = 0;
                        if (k < cnt && i < n && act) {
                            const uint32_t fl = *reinterpret_cast<const uint32_t*>(sr + k);
                            if ((fl & 0xc0c0c0c0u) == 0) {   // no plastic target, no bias: the common quad
                                AccT x[4];
                                load4(sacc + k, x);
                                const float4 v4 = *reinterpret_cast<const float4*>(sv + k);
                                const float4 g4 = *reinterpret_cast<const float4*>(sg + k);
                                float vv[4] = {v4.x, v4.y, v4.z, v4.w}, gg[4] = {g4.x, g4.y, g4.z, g4.w};
                                uint32_t ff = fl;
    #pragma unroll
                                for (int j = 0; j < 4; j++) {          // padding pairs run too; their spikes
                                    int r = (int)((fl >> (8 * j)) & 0x3f);   // are masked below, their state unused
                                    // the engine always fuses the two multiply-adds, as the shipped reference does
                                    if (lif_step<float>(vv[j], gg[j], r, acc_to_real<float>(x[j], L.w_syn), false, 0.0f,
                                                        (kick4 >> j) & 1u, L, n_ref, true))
                                        spk4 |= 1u << j;
                                    ff = (ff & ~(0xffu << (8 * j))) | ((uint32_t)r << (8 * j));
                                }
                                if (i + 4 > n) spk4 &= (1u << (n - i)) - 1u;
                                *reinterpret_cast<float4*>(sv + k) = make_float4(vv[0], vv[1], vv[2], vv[3]);
                                *reinterpret_cast<float4*>(sg + k) = make_float4(gg[0], gg[1], gg[2], gg[3]);
                                *reinterpret_cast<uint32_t*>(sr + k) = ff;
                            } else {
                                const int32_t b = b0 + bl;
                                int64_t* pring_row =
                                    PLASTIC ? S.pring + (pos_mod(t, N.R_pl) * N.B + b) * (int64_t)N.n_ppost : nullptr;
                                // staged quads are advanced after the loop; the rest (a CTA with more
                                // than MAX_SPECIAL of them) out of line here
                                if (!all_staged)
                                    spk4 = quad_special<AccT, PLASTIC>(sacc + k, sv + k, sg + k, sr + k, kick4,
                                                                       min(4, n - i), pring_row, N.ppost_of + i,
                                                                       S.bias_ext + (int64_t)b * S.n_ext, S.ext_idx + i, L,
                                                                       n_ref);
                            }
                        }
                        // the 8 lanes of a 32-pair word OR their nibbles together; one of them stores it
                        uint32_t word = spk4 << sh;
                        word |= __shfl_xor_sync(0xffffffffu, word, 1);
                        word |= __shfl_xor_sync(0xffffffffu, word, 2);
                        word |= __shfl_xor_sync(0xffffffffu, word, 4);
                        if ((lane & 7) == 0) map[k >> 5] = word;
                        i += 4 * U_THREADS;
                        if (i >= np) {
                            do { i -= np; bl++; } while (i >= np);
                            act = bl < 64 && s_active[bl];
                        }
                    }
                    // the staged neurons' plastic deltas of this step, for the listing warps
                    if (tid < 4 * n_sp) {
                        s_sp_pl[(s & 1) * 4 * MAX_SPECIAL + tid] = sp_pl;
                        if (sp_pl != 0) *sp_pl_at = 0;
                    }
                }

                    fence_proxy_async_shared();      // reads of the slice before the next bulk load
                    // the next step's slice, when it lies in this epoch (its arrivals are complete),
                    // loads while this step ends
                    staged = ok && s + 1 < ep1;
                    if (staged) {
                        u_sync();
                        if (tid == 0 && cnt > 0) issue_slice(acc_slot<AccT>(N, S, t + 1) + acc_base, sacc, acc_bytes, mbar);
                    }
                    if (tid == 0) stamp(A, s, 3);
                } else {
                    // ---- the previous step's staged neurons, then its spikes: counts, plastic rows,
                    //      work items --------------------------------------------------------------
                    if (s >= 1 && n_sp > 0) {
                        if (lt < 4 * n_sp) advance_staged(s - 1, t - 1, lt);
                        list_sync();
                    }
                    if (s >= 1)
                        list_spikes<PLASTIC, RECORD>(N, S, A, maps + ((s - 1) % 3) * wpm, s - 1, t - 1, b0, q, lo,
                                                     used_words, s_cnt, s_scan, s_spk, lt, LIST_THREADS,
                                                     []() { list_sync(); });
                    if (lt == 0) stamp(A, s, 8);
                }
            }
        }
        pushed = max(pushed, pa1);
        staged = false;
        if (tid < 32 && cnt > 0) {
            bulk_wait_all();                     // the cleared slices are written before anyone pushes into them
            fence_proxy_async_global();
        }
        if (tid == 0) stamp(A, ep1 - 1, 5);
        barriers++;
        last = ep1 - 1;
        if (grid_barrier(A, barriers * gridDim.x, err, ep1 + 1)) { last = -1; stop = true; break; }
        if (tid == 0) stamp(A, ep1 - 1, 6);
    }
    if (tid < 32) bulk_wait_all();
    // the last step's staged neurons and spikes are settled before the launch ends (the next launch
    // scatters the spikes)
    if (last >= 0 && n_sp > 0) {
        if (tid < 4 * n_sp) advance_staged(last, A.t0 + last, tid);
        __syncthreads();
    }
    if (last >= 0)
        list_spikes<PLASTIC, RECORD>(N, S, A, maps + (last % 3) * wpm, last, A.t0 + last, b0, q, lo, used_words, s_cnt,
                                     s_scan, s_spk, tid, PT, []() { __syncthreads(); });

    // ---- write the state back ------------------------------------------------------------------
    __syncthreads();
    for (int32_t k = tid; k < cnt; k += PT) {
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
inline PersistPlan plan_persistent(int64_t n, int64_t n_pad, int32_t B, bool f64, int n_ref, int n_delay,
                                   int acc_bytes, int sm_count, int device)
{
    PersistPlan P{};
    if (f64 || n_ref > 63 || n_delay < 3) return P;
    int smem_optin = 0;
    cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    if (smem_optin <= 0) smem_optin = 232448;
    int64_t per_max = 0;
    for (int64_t lo = 16, hi = (int64_t)1 << 18; lo <= hi;) {     // largest `per` whose layout fits
        const int64_t mid = (lo + hi) / 2 / 16 * 16;
        if (mid < 16) break;
        if (PersistSmem(mid, acc_bytes).total <= smem_optin) { per_max = mid; lo = mid + 16; }
        else hi = mid - 16;
    }
    if (per_max <= 0) return P;
    const int ctas = sm_count;
    int64_t gmax = std::min<int64_t>((int64_t)ctas * per_max / n_pad, 63);
    if (gmax < 1) return P;
    const int32_t n_groups = (int32_t)((B + gmax - 1) / gmax);
    const int32_t G = (B + n_groups - 1) / n_groups;
    int64_t per = ((int64_t)G * n_pad + ctas - 1) / ctas;
    per = (per + 15) / 16 * 16;
    if (per > per_max || per >= ((int64_t)1 << 18) || ctas > MAX_SEG) return P;
    P.group = G;
    P.n_groups = n_groups;
    P.ctas = ctas;
    P.per = per;
    P.smem = (size_t)PersistSmem(per, acc_bytes).total;
    P.launches_per_run = n_groups;
    (void)n;
    return P;
}

template <typename AccT, bool RASTER, int PLASTIC, bool RECORD, int LANES>
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

template <typename AccT, bool RASTER, int PLASTIC, bool RECORD>
cudaError_t launch_persist_lanes(const PersistPlan& P, const DevNet& N, const DevState& S, const PersistArgs& A,
                                 int lanes, cudaStream_t st)
{
    if (lanes == 8) return launch_persist_one<AccT, RASTER, PLASTIC, RECORD, 8>(P, N, S, A, st);
    if (lanes == 16) return launch_persist_one<AccT, RASTER, PLASTIC, RECORD, 16>(P, N, S, A, st);
    return launch_persist_one<AccT, RASTER, PLASTIC, RECORD, 32>(P, N, S, A, st);
}

// plastic: 0 none, 1 plastic synapses, 2 plastic synapses in long rows (several per presynaptic
// neuron: their pushes batched); the batched form only without a kick raster or per-step records
template <typename AccT>
cudaError_t launch_persist_acc(const PersistPlan& P, const DevNet& N, const DevState& S, const PersistArgs& A,
                               int plastic, bool raster, bool record, int lanes, cudaStream_t st)
{
#define LP_(R_, P_, C_) return launch_persist_lanes<AccT, R_, P_, C_>(P, N, S, A, lanes, st)
    if (raster) {
        if (plastic) { if (record) LP_(true, 1, true); LP_(true, 1, false); }
        if (record) LP_(true, 0, true);
        LP_(true, 0, false);
    }
    if (plastic) {
        if (record) LP_(false, 1, true);
        if (plastic == 2) LP_(false, 2, false);
        LP_(false, 1, false);
    }
    if (record) LP_(false, 0, true);
    LP_(false, 0, false);
#undef LP_
}

inline cudaError_t launch_persistent(const PersistPlan& P, const DevNet& N, const DevState& S, const PersistArgs& A,
                                     int acc_mode, int plastic, bool raster, bool record, int lanes, cudaStream_t st)
{
    if (acc_mode == 0) return launch_persist_acc<int32_t>(P, N, S, A, plastic, raster, record, lanes, st);
    return launch_persist_acc<int64_t>(P, N, S, A, plastic, raster, record, lanes, st);
}

}  // namespace fb
