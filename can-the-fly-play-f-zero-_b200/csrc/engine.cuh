// Device-resident layout of one engine (a connectome shared by B instances) and the
// two-launches-per-step kernels. Layout in HBM:
//
//   connectome  rowptr[n+1] i64 (rows padded to 8 entries), col[nnz_pad] i32,
//               cnt[nnz_pad] i16 (INT32 mode) or wfx[nnz_pad] i64 (Q32.32 mode)
//   plastic     pl_rowptr[n+1] i64 (by presynaptic neuron), pl_pidx[n_pl] i32 (compact target),
//               pl_q0[n_pl] i64, ppost_of[n] i32 (compact target index or -1), pw[B][n_pl] f32.
//               Plastic entries keep their connectome weight in the fixed CSR; an instance's
//               weight pw enters as the Q32.32 delta q32(pw) - q32(w0), pushed at spike time.
//   state       v[B][n], g[B][n] (f32 or f64), ref[B][n] i8
//   inputs      ext_idx[n] i32, p_ext[B][n_ext] f32, bias_ext[B][n_ext] f32
//   delay line  acc[S][B][n_pad] (i32 or i64): synaptic input of the next S ticks (slot = tick mod
//               S, S = 2 x the persistent engine's epoch, at least 2), rows padded to 16 entries so
//               that every row starts on a 64-byte boundary (TMA bulk copies);
//               items[R][n_groups][n_seg][cap_c] int2: spike work lists of the last R = n_delay+1
//               steps, one per instance group and segment (the pairs one persistent CTA owns);
//               item_count[R][n_groups][n_seg]; pring[R_pl][B][n_ppost] i64: plastic input (R_pl = n_delay + epoch: a slot
//               is cleared by its reader at least one epoch before anyone pushes into it again);
//               with pull propagation also masks[R][n][ceil(B/64)] u64: which instances each
//               neuron spiked in, and the connectome by postsynaptic neuron (colptr, cpre, ccnt/cwfx)
//
// The delay line is "deferred push": the fixed-weight rows of the spikes of step s are scattered
// into acc only shortly before they arrive (the step engine at step s + n_delay - 1, the
// persistent engine one epoch ahead), so only S accumulator slots (instead of n_delay) are live. Fixed weights never change during a run and integer addition is
// order-free, so this equals the reference's push-at-spike-time ring (brain.py:54-56) exactly.
// Plastic weights may change between runs, so their rows are pushed at spike time.
#pragma once
#include "common.cuh"

namespace fb {

struct DevNet {
    int64_t n, n_pad;
    int32_t B, n_delay, R, n_ref;
    int32_t R_pl;              // plastic input ring slots: n_delay + the persistent engine's epoch
    const int64_t* rowptr;
    const int32_t* col;
    const int16_t* cnt;
    const int64_t* wfx;
    int64_t n_pl;
    int32_t n_ppost;
    const int64_t* pl_rowptr;
    const int32_t* pl_pidx;
    const int64_t* pl_q0;      // q32 of each plastic entry's connectome weight
    const int32_t* ppost_of;
    const int64_t* colptr;     // pull propagation: the connectome by postsynaptic neuron (or nullptr)
    const int32_t* cpre;
    const int16_t* ccnt;
    const int64_t* cwfx;
    Lif<float> L32;
    Lif<double> L64;
};

struct DevState {
    void* v;
    void* g;
    int8_t* ref;
    const float* pw;
    const int32_t* ext_idx;
    int32_t n_ext;
    const float* p_ext;
    const float* bias_ext;
    void* acc;                 // [n_slots][B][n_pad]
    int32_t n_slots;
    int64_t* pring;
    int2* items;               // [R][n_groups][n_seg][cap_c]
    int32_t* item_count;       // [R][n_groups][n_seg]
    int64_t cap_c;             // items per (step, group, segment) list
    int32_t group;             // instances per group (group of instance b = b / group)
    int32_t n_groups;
    int32_t n_seg;             // segments per group: the CTAs of the persistent plan (1 without one)
    int64_t seg_pairs;         // pairs per segment; pair (b, i) = (b mod group) * n_pad + i
    const int64_t* reset_tick;
    const int64_t* stop_tick;
    unsigned long long* masks; // pull propagation: [R][n][mask_words] spiking instances per neuron (or nullptr)
    int32_t mask_words;        // ceil(B / 64)
    int32_t* err;              // [0] overflow, [1] barrier timeout step (host-mapped)
    uint32_t seed;
};

struct StepArgs {
    int64_t t;                 // tick of this step
    uint32_t step_no;          // Poisson hash counter
    int32_t s;                 // index of this step within the run
    const uint32_t* kicks;     // raster of this run or nullptr
    int32_t words;             // raster words per instance-step
    int32_t* counts;           // (B, n) this run's counts
    int32_t* step_counts;      // (steps, B) or nullptr
    uint64_t* step_digest;     // (steps, B) or nullptr
};

__device__ __forceinline__ int64_t pos_mod(int64_t a, int64_t m) { int64_t r = a % m; return r < 0 ? r + m : r; }

__device__ __forceinline__ bool bits_differ(float a, float b) { return __float_as_uint(a) != __float_as_uint(b); }
__device__ __forceinline__ bool bits_differ(double a, double b)
{
    return __double_as_longlong(a) != __double_as_longlong(b);
}

// accumulator slot of tick t
template <typename AccT> __device__ __forceinline__ AccT* acc_slot(const DevNet& N, const DevState& S, int64_t t)
{
    return reinterpret_cast<AccT*>(S.acc) + pos_mod(t, S.n_slots) * (int64_t)N.B * N.n_pad;
}

template <typename Real> __device__ __forceinline__ const Lif<Real>& lif_of(const DevNet& N);
template <> __device__ __forceinline__ const Lif<float>& lif_of<float>(const DevNet& N) { return N.L32; }
template <> __device__ __forceinline__ const Lif<double>& lif_of<double>(const DevNet& N) { return N.L64; }

__device__ __forceinline__ int2* list_of(const DevState& S, int64_t slot, int32_t q, int32_t c)
{
    return S.items + (((int64_t)slot * S.n_groups + q) * S.n_seg + c) * S.cap_c;
}
__device__ __forceinline__ int32_t* count_of(const DevState& S, int64_t slot, int32_t q, int32_t c)
{
    return S.item_count + ((int64_t)slot * S.n_groups + q) * S.n_seg + c;
}
// list key (group * n_seg + segment) of the pair (b, i)
__device__ __forceinline__ int32_t list_key(const DevState& S, int64_t n_pad, int32_t b, int32_t i)
{
    const int32_t q = b / S.group;
    const int64_t p = (int64_t)(b - q * S.group) * n_pad + i;
    return q * S.n_seg + (int32_t)(p / S.seg_pairs);
}

// Fire-and-forget reductions into global memory (no value comes back; the address is converted to
// the global window explicitly, so the hardware never falls back to a returning generic atomic).
// No "memory" clobber: the reduced words are never read in the phase that reduces into them, and
// leaving the clobber out lets the compiler issue the next edges' loads before these reductions.
__device__ __forceinline__ void red_add(int32_t* p, int32_t x)
{
    asm volatile("red.relaxed.gpu.global.add.s32 [%0], %1;" ::"l"(__cvta_generic_to_global(p)), "r"(x));
}
__device__ __forceinline__ void red_add(int64_t* p, int64_t x)
{
    asm volatile("red.relaxed.gpu.global.add.u64 [%0], %1;" ::"l"(__cvta_generic_to_global(p)), "l"(x));
}

// A work item: up to CHUNK consecutive entries of a spiking row, {first entry in the padded CSR,
// (instance << CHUNK_BITS) | number of entries}.
__device__ __forceinline__ int2 make_item(const DevNet& N, int32_t i, int32_t b, int c)
{
    const int64_t r0 = N.rowptr[i], r1 = N.rowptr[i + 1];
    const int64_t k0 = r0 + (int64_t)c * CHUNK;
    return make_int2((int32_t)k0, (b << CHUNK_BITS) | (int32_t)min((int64_t)CHUNK, r1 - k0));
}

// Append `nch` work items (this lane's spike: chunks 0..nch-1 of row i of instance b) to the list of
// the lane's (group, segment); one atomic per warp and list (the ballot/shuffle compaction).
__device__ __forceinline__ void warp_append(const DevNet& N, const DevState& S, int64_t slot, int nch, int32_t i,
                                            int32_t b)
{
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    unsigned todo = __ballot_sync(FULL, nch > 0);
    if (!todo) return;
    const int32_t key = nch > 0 ? list_key(S, N.n_pad, b, i) : -1;
    while (todo) {
        const int leader = __ffs(todo) - 1;
        const int32_t kk = __shfl_sync(FULL, key, leader);
        const bool mine = nch > 0 && key == kk;
        int incl = mine ? nch : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += y;
        }
        const int total = __shfl_sync(FULL, incl, 31);
        const int32_t q = kk / S.n_seg, c = kk - q * S.n_seg;
        int base = 0;
        if (lane == 31) base = atomicAdd(count_of(S, slot, q, c), total);
        base = __shfl_sync(FULL, base, 31);
        if (mine) {
            int2* list = list_of(S, slot, q, c);
            const int64_t start = (int64_t)base + incl - nch;
            for (int ch = 0; ch < nch; ch++) {
                const int64_t p = start + ch;
                if (p < S.cap_c) list[p] = make_item(N, i, b, ch);
                else atomicExch(S.err, 1);
            }
        }
        todo &= ~__ballot_sync(FULL, mine);
    }
}

// Plastic row of a spiking neuron, pushed at spike time into the ring slot it arrives from.
__device__ __forceinline__ void push_plastic_row(const DevNet& N, const DevState& S, int64_t t, int32_t b, int32_t i)
{
    const int64_t p0 = N.pl_rowptr[i], p1 = N.pl_rowptr[i + 1];
    if (p0 == p1) return;
    unsigned long long* dst = reinterpret_cast<unsigned long long*>(
        S.pring + (pos_mod(t + N.n_delay, N.R_pl) * N.B + b) * (int64_t)N.n_ppost);
    const float* w = S.pw + (int64_t)b * N.n_pl;
    for (int64_t k = p0; k < p1; k++) {
        const int64_t d = to_q32(w[k]) - N.pl_q0[k];
        if (d != 0) red_add(reinterpret_cast<int64_t*>(dst) + N.pl_pidx[k], d);
    }
}

// The same for networks whose plastic rows are long (several plastic synapses per presynaptic
// neuron): four entries at a time, their loads in flight together, then their reductions (a
// reduction between two loads keeps the second from being issued early). Same sums.
__device__ __forceinline__ void push_plastic_row_batched(const DevNet& N, const DevState& S, int64_t t, int32_t b,
                                                         int32_t i)
{
    const int64_t p0 = N.pl_rowptr[i], p1 = N.pl_rowptr[i + 1];
    if (p0 == p1) return;
    int64_t* dst = S.pring + (pos_mod(t + N.n_delay, N.R_pl) * N.B + b) * (int64_t)N.n_ppost;
    const float* w = S.pw + (int64_t)b * N.n_pl;
    for (int64_t k0 = p0; k0 < p1; k0 += 4) {
        float wv[4];
        int64_t q0[4];
        int32_t pi[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int64_t k = min(k0 + u, p1 - 1);
            wv[u] = w[k];
            q0[u] = N.pl_q0[k];
            pi[u] = N.pl_pidx[k];
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int64_t d = to_q32(wv[u]) - q0[u];
            if (k0 + u < p1 && d != 0) red_add(dst + pi[u], d);
        }
    }
}

// Arriving plastic input of (b, i) at tick t, read and cleared (L2 only: other SMs wrote it).
template <typename Real>
__device__ __forceinline__ Real take_plastic(const DevNet& N, const DevState& S, int64_t t, int32_t b, int32_t i)
{
    const int32_t pp = N.ppost_of[i];
    int64_t* q = S.pring + (pos_mod(t, N.R_pl) * N.B + b) * (int64_t)N.n_ppost + pp;
    const int64_t px = __ldcg(reinterpret_cast<const long long*>(q));
    if (px != 0) *q = 0;
    return from_q32<Real>(px);
}

// Poisson kick of ext slot j of instance b at run step s (raster) or hash draw.
template <bool RASTER>
__device__ __forceinline__ bool kick_of(const DevState& S, const uint32_t* kicks, int32_t words, int32_t B, int32_t s,
                                        int32_t b, int32_t j, uint32_t tid, uint32_t step_no)
{
    if (RASTER) {
        const uint32_t w = kicks[((int64_t)s * B + b) * words + (j >> 5)];
        return (w >> (j & 31)) & 1u;
    }
    const float p = S.p_ext[(int64_t)b * S.n_ext + j];
    return p > 0.0f && hash_kick(tid, step_no, S.seed, (uint32_t)b, p);
}

// ---------------------------------------------------------------------------------------------
// Step engine, kernel 1: every (instance, neuron) advances one step; spikes become work items.
// ---------------------------------------------------------------------------------------------
template <typename Real, typename AccT, bool RASTER, bool PLASTIC, bool RECORD>
__global__ void __launch_bounds__(256) k_update(const DevNet N, const DevState S, const StepArgs A)
{
    const int64_t n = N.n;
    const int64_t total = (int64_t)N.B * n;
    const Lif<Real>& L = lif_of<Real>(N);
    const int64_t t = A.t;
    if (blockIdx.x == 0)       // the lists consumed by the push at t-1 start empty again
        for (int32_t k = threadIdx.x; k < S.n_groups * S.n_seg; k += blockDim.x)
            S.item_count[pos_mod(t - N.n_delay, N.R) * S.n_groups * S.n_seg + k] = 0;
    AccT* acc = acc_slot<AccT>(N, S, t);
    Real* V = reinterpret_cast<Real*>(S.v);
    Real* G = reinterpret_cast<Real*>(S.g);
    const int64_t slot = pos_mod(t, N.R);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < total; base += stride) {
        const int64_t pair = base + threadIdx.x;
        int nch = 0;
        int32_t b = 0, i = 0;
        if (pair < total) {
            b = (int32_t)(pair / n);
            i = (int32_t)(pair - (int64_t)b * n);
            if (t < S.stop_tick[b]) {
                AccT* ap = acc + (int64_t)b * N.n_pad + i;
                const AccT x = *ap;
                if (x != 0) *ap = 0;
                Real buf = acc_to_real<Real>(x, L.w_syn);
                if (PLASTIC && N.ppost_of[i] >= 0) buf = add_rn(buf, take_plastic<Real>(N, S, t, b, i));
                Real v = V[pair], g = G[pair];
                const Real v0 = v, g0 = g;
                const int r0 = S.ref[pair];
                int r = r0;
                const int32_t j = S.ext_idx[i];
                float bias = 0.0f;
                bool kicked = false;
                if (j >= 0) {
                    bias = S.bias_ext[(int64_t)b * S.n_ext + j];
                    kicked = kick_of<RASTER>(S, A.kicks, A.words, N.B, A.s, b, j, (uint32_t)pair, A.step_no);
                }
                // the engine always fuses the two multiply-adds, as the shipped reference kernel does
                const bool spk = lif_step<Real>(v, g, r, buf, j >= 0, bias, kicked, L, N.n_ref, true);
                if (bits_differ(g, g0)) G[pair] = g;
                if (bits_differ(v, v0)) V[pair] = v;
                if (r != r0) S.ref[pair] = (int8_t)r;
                if (spk) {
                    A.counts[pair] += 1;
                    if (S.masks)
                        atomicOr(S.masks + (slot * n + i) * S.mask_words + (b >> 6), 1ull << (b & 63));
                    const int64_t len = N.rowptr[i + 1] - N.rowptr[i];
                    nch = (int)((len + CHUNK - 1) / CHUNK);
                    if (PLASTIC) push_plastic_row(N, S, t, b, i);
                    if (RECORD) {
                        if (A.step_counts) atomicAdd(A.step_counts + (int64_t)A.s * N.B + b, 1);
                        if (A.step_digest)
                            atomicAdd(reinterpret_cast<unsigned long long*>(A.step_digest + (int64_t)A.s * N.B + b),
                                      (unsigned long long)spike_tag((uint64_t)i));
                    }
                }
            }
        }
        warp_append(N, S, slot, nch, i, b);
    }
}

// 8 consecutive CSR entries of one lane: weights (one or four 16-byte loads) and columns (two).
template <typename AccT> struct Edges8;
template <> struct Edges8<int32_t> {
    int32_t w[8];
    int32_t c[8];
    __device__ __forceinline__ void load(const DevNet& N, int64_t k)
    {
        const int4 cw = __ldg(reinterpret_cast<const int4*>(N.cnt + k));
        const int4 c0 = __ldg(reinterpret_cast<const int4*>(N.col + k));
        const int4 c1 = __ldg(reinterpret_cast<const int4*>(N.col + k + 4));
        const uint32_t u[4] = {(uint32_t)cw.x, (uint32_t)cw.y, (uint32_t)cw.z, (uint32_t)cw.w};
#pragma unroll
        for (int q = 0; q < 4; q++) {
            w[2 * q] = (int32_t)(int16_t)(u[q] & 0xffffu);
            w[2 * q + 1] = (int32_t)(int16_t)(u[q] >> 16);
        }
        c[0] = c0.x; c[1] = c0.y; c[2] = c0.z; c[3] = c0.w;
        c[4] = c1.x; c[5] = c1.y; c[6] = c1.z; c[7] = c1.w;
    }
};
template <> struct Edges8<int64_t> {
    int64_t w[8];
    int32_t c[8];
    __device__ __forceinline__ void load(const DevNet& N, int64_t k)
    {
        const longlong2* p = reinterpret_cast<const longlong2*>(N.wfx + k);
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const longlong2 x = __ldg(p + q);
            w[2 * q] = x.x;
            w[2 * q + 1] = x.y;
        }
        const int4 c0 = __ldg(reinterpret_cast<const int4*>(N.col + k));
        const int4 c1 = __ldg(reinterpret_cast<const int4*>(N.col + k + 4));
        c[0] = c0.x; c[1] = c0.y; c[2] = c0.z; c[3] = c0.w;
        c[4] = c1.x; c[5] = c1.y; c[6] = c1.z; c[7] = c1.w;
    }
};

// Scatter one work item (<= CHUNK entries of a spiking row) with LANES lanes, 8 entries a lane.
template <typename AccT, int LANES>
__device__ __forceinline__ void push_item(const DevNet& N, AccT* acc_b, int64_t k0, int32_t len, int lane)
{
    const int64_t k1 = k0 + len;
#pragma unroll 2
    for (int64_t k = k0 + (int64_t)lane * 8; k < k1; k += LANES * 8) {
        Edges8<AccT> e;
        e.load(N, k);
#pragma unroll
        for (int q = 0; q < 8; q++)
            if (e.w[q] != 0) red_add(acc_b + e.c[q], e.w[q]);
    }
}

// Inclusive prefix over the n_seg segment counts of list (slot, q) into `pre` (shared memory),
// computed by one warp (n_seg <= MAX_SEG); returns the total. Counts are clamped to the capacity.
constexpr int MAX_SEG = 256;
__device__ __forceinline__ int32_t segment_prefix(const DevState& S, int64_t slot, int32_t q, int32_t* pre)
{
    constexpr int PER_LANE = MAX_SEG / 32;
    const int lane = threadIdx.x & 31;
    const int32_t* cnt = count_of(S, slot, q, 0);
    const int32_t c0 = lane * PER_LANE;
    int32_t x[PER_LANE];
#pragma unroll
    for (int j = 0; j < PER_LANE; j++) x[j] = c0 + j < S.n_seg ? __ldcg(cnt + c0 + j) : 0;   // all in flight
    int32_t sum = 0;
#pragma unroll
    for (int j = 0; j < PER_LANE; j++) {
        x[j] = (int32_t)min((int64_t)max(x[j], 0), S.cap_c);
        sum += x[j];
    }
    int32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    int32_t run = incl - sum;
#pragma unroll
    for (int j = 0; j < PER_LANE; j++) {
        run += x[j];
        if (c0 + j < S.n_seg) pre[c0 + j] = run;
    }
    return __shfl_sync(0xffffffffu, incl, 31);
}

// Scatter the items [g0, g1) of list (slot of spike step s = t+1-n_delay, group q) into acc_next.
// The list is the concatenation of its segments, described by their inclusive prefix `pre`; lane
// group `lg` of `n_lg` (LANES lanes each, lane `lane` within it) takes items g0+lg, g0+lg+n_lg, ...
// and follows the segment boundaries forward (a search only when it crosses one). Items of
// instance b are skipped unless reset_tick[b - b_base] <= s and t+1 < stop_tick[b - b_base].
template <typename AccT, int LANES>
__device__ __forceinline__ void push_range(const DevNet& N, const DevState& S, int64_t t, int32_t q, AccT* acc_next,
                                           const int32_t* pre, int64_t g0, int64_t g1, int64_t lg, int64_t n_lg,
                                           int lane, const int64_t* reset_tick, const int64_t* stop_tick,
                                           int32_t b_base)
{
    const int64_t s = t + 1 - N.n_delay;
    if (s < 0) return;
    const int64_t slot = pos_mod(s, N.R);
    int32_t seg = -1;
    int64_t seg_lo = 0, seg_hi = 0;
    for (int64_t g = g0 + lg; g < g1; g += n_lg) {
        if (g >= seg_hi) {                        // first segment whose prefix exceeds g
            int32_t lo = seg + 1, hi = S.n_seg - 1;
            while (lo < hi) {
                const int32_t mid = (lo + hi) >> 1;
                if (pre[mid] > g) hi = mid;
                else lo = mid + 1;
            }
            seg = lo;
            seg_lo = lo > 0 ? pre[lo - 1] : 0;
            seg_hi = pre[lo];
        }
        const int2 item = __ldcg(list_of(S, slot, q, seg) + (g - seg_lo));
        const int32_t b = item.y >> CHUNK_BITS;
        if (s < reset_tick[b - b_base] || t + 1 >= stop_tick[b - b_base]) continue;
        push_item<AccT, LANES>(N, acc_next + (int64_t)b * N.n_pad, (int64_t)(uint32_t)item.x,
                               item.y & ((1 << CHUNK_BITS) - 1), lane);
    }
}

// ---------------------------------------------------------------------------------------------
// Step engine, kernel 2: the spikes of step t+1-n_delay (they arrive at step t+1) are scattered
// into the accumulator that step t+1 reads; each block takes a contiguous share of every list.
// ---------------------------------------------------------------------------------------------
// The spike-mask slot that step t+1 records into starts empty (it last held step t-n_delay, whose
// propagation ran at step t-1).
__device__ __forceinline__ void clear_mask_slot(const DevNet& N, const DevState& S, int64_t t)
{
    if (!S.masks) return;
    const int64_t words = N.n * S.mask_words;
    unsigned long long* m = S.masks + pos_mod(t + 1, N.R) * words;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < words; k += (int64_t)gridDim.x * blockDim.x)
        m[k] = 0ull;
}

// `do_push` 0: the arrivals of t+1 were pushed ahead already (by the persistent engine); only the
// mask slot is cleared.
template <typename AccT, int LANES>
__global__ void __launch_bounds__(256) k_push(const DevNet N, const DevState S, int64_t t, int do_push)
{
    __shared__ int32_t pre[MAX_SEG];
    __shared__ int32_t s_total;
    clear_mask_slot(N, S, t);
    if (!do_push || t + 1 - N.n_delay < 0) return;
    AccT* acc = acc_slot<AccT>(N, S, t + 1);
    const int64_t slot = pos_mod(t + 1 - N.n_delay, N.R);
    for (int32_t q = 0; q < S.n_groups; q++) {
        if (threadIdx.x < 32) {
            const int32_t tot = segment_prefix(S, slot, q, pre);
            if (threadIdx.x == 0) s_total = tot;
        }
        __syncthreads();
        const int64_t total = s_total;
        const int64_t g0 = total * blockIdx.x / gridDim.x, g1 = total * (blockIdx.x + 1) / gridDim.x;
        push_range<AccT, LANES>(N, S, t, q, acc, pre, g0, g1, threadIdx.x / LANES, blockDim.x / LANES,
                                threadIdx.x % LANES, S.reset_tick, S.stop_tick, 0);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------
// Pull propagation (step engine, kernel 2 alternative): every postsynaptic neuron j gathers its
// incoming entries whose presynaptic neuron spiked at step s = t+1-n_delay, for the instances of
// one 64-bit mask word per thread. The sums are exact integers, so push and pull give identical
// accumulators; pull reads the whole connectome once per step for all instances, push only the
// rows of the spikes (it pays off only when a large share of neurons fires every step).
// ---------------------------------------------------------------------------------------------
template <typename AccT> __device__ __forceinline__ AccT pull_weight(const DevNet& N, int64_t e);
template <> __device__ __forceinline__ int32_t pull_weight<int32_t>(const DevNet& N, int64_t e) { return N.ccnt[e]; }
template <> __device__ __forceinline__ int64_t pull_weight<int64_t>(const DevNet& N, int64_t e) { return N.cwfx[e]; }

template <typename AccT>
__global__ void __launch_bounds__(256) k_pull(const DevNet N, const DevState S, int64_t t)
{
    clear_mask_slot(N, S, t);
    const int64_t s = t + 1 - N.n_delay;
    if (s < 0) return;
    AccT* acc = acc_slot<AccT>(N, S, t + 1);
    const int W = S.mask_words;
    const unsigned long long* M = S.masks + pos_mod(s, N.R) * N.n * W;
    const int64_t total = N.n * W;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < total; p += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = p / W;
        const int w = (int)(p - j * W);
        const int64_t e1 = N.colptr[j + 1];
        for (int64_t e = N.colptr[j]; e < e1; e++) {
            unsigned long long m = __ldg(M + (int64_t)N.cpre[e] * W + w);
            if (!m) continue;
            const AccT c = pull_weight<AccT>(N, e);
            while (m) {
                const int32_t b = w * 64 + __ffsll((long long)m) - 1;
                m &= m - 1;
                if (s < S.reset_tick[b] || t + 1 >= S.stop_tick[b]) continue;
                acc[(int64_t)b * N.n_pad + j] += c;     // (b, j) belongs to this thread alone
            }
        }
    }
}

}  // namespace fb
