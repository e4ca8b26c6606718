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
//   delay line  acc[2][B][n_pad] (i32 or i64): synaptic input of the next two steps, rows padded
//               to 16 entries so that every row starts on a 64-byte boundary (TMA bulk copies);
//               items[R][n_groups][cap_g] int2: spike work lists of the last R = n_delay+1 steps,
//               one list per instance group; pring[R][B][n_ppost] i64: plastic input
//
// The delay line is "deferred push": the fixed-weight rows of the spikes of step s are scattered
// into acc only at step s + n_delay - 1, right before they arrive, so only two accumulator slots
// (instead of n_delay) are live. Fixed weights never change during a run and integer addition is
// order-free, so this equals the reference's push-at-spike-time ring (brain.py:54-56) exactly.
// Plastic weights may change between runs, so their rows are pushed at spike time.
#pragma once
#include "common.cuh"

namespace fb {

struct DevNet {
    int64_t n, n_pad;
    int32_t B, n_delay, R, n_ref;
    int32_t contract;
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
    void* acc0;
    void* acc1;
    int64_t* pring;
    int2* items;
    int32_t* item_count;       // [R][n_groups]
    int64_t cap_g;             // items per (step, group) list
    int32_t group;             // instances per group (list owner = b / group)
    int32_t n_groups;
    const int64_t* reset_tick;
    const int64_t* stop_tick;
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

template <typename Real> __device__ __forceinline__ const Lif<Real>& lif_of(const DevNet& N);
template <> __device__ __forceinline__ const Lif<float>& lif_of<float>(const DevNet& N) { return N.L32; }
template <> __device__ __forceinline__ const Lif<double>& lif_of<double>(const DevNet& N) { return N.L64; }

__device__ __forceinline__ int2* list_of(const DevState& S, int64_t slot, int32_t q)
{
    return S.items + ((int64_t)slot * S.n_groups + q) * S.cap_g;
}
__device__ __forceinline__ int32_t* count_of(const DevState& S, int64_t slot, int32_t q)
{
    return S.item_count + (int64_t)slot * S.n_groups + q;
}

// A work item: up to CHUNK consecutive entries of a spiking row, {first entry in the padded CSR,
// (instance << CHUNK_BITS) | number of entries}.
__device__ __forceinline__ int2 make_item(const DevNet& N, int32_t i, int32_t b, int c)
{
    const int64_t r0 = N.rowptr[i], r1 = N.rowptr[i + 1];
    const int64_t k0 = r0 + (int64_t)c * CHUNK;
    return make_int2((int32_t)k0, (b << CHUNK_BITS) | (int32_t)min((int64_t)CHUNK, r1 - k0));
}

// Append `nch` work items (this lane's spike: chunks 0..nch-1 of row i of instance b) to the list
// of the lane's instance group; one atomic per warp and group (the ballot/shuffle compaction).
__device__ __forceinline__ void warp_append(const DevNet& N, const DevState& S, int64_t slot, int nch, int32_t i,
                                            int32_t b)
{
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    unsigned todo = __ballot_sync(FULL, nch > 0);
    const int32_t q = b / S.group;
    while (todo) {
        const int leader = __ffs(todo) - 1;
        const int32_t qq = __shfl_sync(FULL, q, leader);
        const bool mine = nch > 0 && q == qq;
        int incl = mine ? nch : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += y;
        }
        const int total = __shfl_sync(FULL, incl, 31);
        int base = 0;
        if (lane == 31) base = atomicAdd(count_of(S, slot, qq), total);
        base = __shfl_sync(FULL, base, 31);
        if (mine) {
            int2* list = list_of(S, slot, qq);
            const int64_t start = (int64_t)base + incl - nch;
            for (int c = 0; c < nch; c++) {
                const int64_t p = start + c;
                if (p < S.cap_g) list[p] = make_item(N, i, b, c);
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
        S.pring + (pos_mod(t + N.n_delay, N.R) * N.B + b) * (int64_t)N.n_ppost);
    const float* w = S.pw + (int64_t)b * N.n_pl;
    for (int64_t k = p0; k < p1; k++) {
        const int64_t d = to_q32(w[k]) - N.pl_q0[k];
        if (d != 0) atomicAdd(dst + N.pl_pidx[k], (unsigned long long)d);
    }
}

// Arriving plastic input of (b, i) at tick t, read and cleared (L2 only: other SMs wrote it).
template <typename Real>
__device__ __forceinline__ Real take_plastic(const DevNet& N, const DevState& S, int64_t t, int32_t b, int32_t i)
{
    const int32_t pp = N.ppost_of[i];
    int64_t* q = S.pring + (pos_mod(t, N.R) * N.B + b) * (int64_t)N.n_ppost + pp;
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
    if (blockIdx.x == 0 && threadIdx.x < S.n_groups)
        *count_of(S, pos_mod(t - N.n_delay, N.R), threadIdx.x) = 0;   // consumed by the push at t-1
    AccT* acc = reinterpret_cast<AccT*>((t & 1) ? S.acc1 : S.acc0);
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
                const bool spk = lif_step<Real>(v, g, r, buf, j >= 0, bias, kicked, L, N.n_ref, N.contract != 0);
                if (bits_differ(g, g0)) G[pair] = g;
                if (bits_differ(v, v0)) V[pair] = v;
                if (r != r0) S.ref[pair] = (int8_t)r;
                if (spk) {
                    A.counts[pair] += 1;
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

__device__ __forceinline__ void red_add(int32_t* p, int32_t x) { atomicAdd(p, x); }
__device__ __forceinline__ void red_add(int64_t* p, int64_t x)
{
    atomicAdd(reinterpret_cast<unsigned long long*>(p), (unsigned long long)x);
}

// Scatter one work item (<= CHUNK entries of a spiking row) with LANES lanes, 8 entries a lane.
template <typename AccT, int LANES>
__device__ __forceinline__ void push_item(const DevNet& N, AccT* acc_b, int64_t k0, int32_t len, int lane)
{
    const int64_t k1 = k0 + len;
    for (int64_t k = k0 + (int64_t)lane * 8; k < k1; k += LANES * 8) {
        Edges8<AccT> e;
        e.load(N, k);
#pragma unroll
        for (int q = 0; q < 8; q++)
            if (e.w[q] != 0) red_add(acc_b + e.c[q], e.w[q]);
    }
}

// Scatter the group-q list of spike step s (arriving at tick t+1) into acc_next, `ngroups_total`
// groups of LANES lanes striding over the items. Lists are read through L2 (other SMs wrote them).
template <typename AccT, int LANES>
__device__ __forceinline__ void push_list(const DevNet& N, const DevState& S, int64_t t, int32_t q, AccT* acc_next,
                                          int64_t gtid, int64_t nthreads)
{
    const int64_t s = t + 1 - N.n_delay;
    if (s < 0) return;
    const int64_t slot = pos_mod(s, N.R);
    const int64_t n_items = min((int64_t)__ldcg(count_of(S, slot, q)), S.cap_g);
    const int2* list = list_of(S, slot, q);
    const int lane = (int)(gtid % LANES);
    const int64_t ngroups = nthreads / LANES;
    for (int64_t it = gtid / LANES; it < n_items; it += ngroups) {
        const int2 item = __ldcg(list + it);
        const int32_t b = item.y >> CHUNK_BITS;
        if (s < S.reset_tick[b] || t + 1 >= S.stop_tick[b]) continue;
        push_item<AccT, LANES>(N, acc_next + (int64_t)b * N.n_pad, (int64_t)(uint32_t)item.x,
                               item.y & ((1 << CHUNK_BITS) - 1), lane);
    }
}

// ---------------------------------------------------------------------------------------------
// Step engine, kernel 2: the spikes of step t+1-n_delay (they arrive at step t+1) are scattered
// into the accumulator that step t+1 reads. LANES lanes per work item.
// ---------------------------------------------------------------------------------------------
template <typename AccT, int LANES>
__global__ void __launch_bounds__(256) k_push(const DevNet N, const DevState S, int64_t t)
{
    AccT* acc = reinterpret_cast<AccT*>(((t + 1) & 1) ? S.acc1 : S.acc0);
    const int64_t gtid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nthreads = (int64_t)gridDim.x * blockDim.x;
    for (int32_t q = 0; q < S.n_groups; q++) push_list<AccT, LANES>(N, S, t, q, acc, gtid, nthreads);
}

}  // namespace fb
