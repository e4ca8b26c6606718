// Host-side preparation of the engine's device layout (pure C++, no CUDA): CSR validation and
// sorting, weight classification, the 8-entry-padded device CSR, and the plastic-entry plan.
// Kept separate so that it can be compiled and checked on a CPU (tests/host_prep_check.cpp).
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

namespace fb {

constexpr int HOST_CHUNK = 256;      // must equal CHUNK in common.cuh
constexpr int HOST_CHUNK_BITS = 12;  // must equal CHUNK_BITS
constexpr int HOST_EDGE_ALIGN = 8;   // must equal EDGE_ALIGN

// float weight -> Q32.32, round half to even (x * 2^32 is exact in double)
inline int64_t q32_host(float w) { return (int64_t)std::llrint((double)w * 4294967296.0); }

struct HostCsr {
    int64_t n = 0, nnz = 0, nnz_pad = 0;
    int acc_mode = 0;                 // 0: int16 counts (INT32 accumulation), 1: Q32.32
    std::vector<int64_t> ip;          // (n+1) row pointers of the caller's CSR
    std::vector<int32_t> ix;          // (nnz) columns, sorted within rows
    std::vector<float> wd;            // (nnz) f32(count * f32(w_syn)) (brain.py:89)
    std::vector<int64_t> rp;          // (n+1) padded row pointers (multiples of 8)
    std::vector<int32_t> pcol;        // (nnz_pad) columns, padding 0
    std::vector<int16_t> pcnt;        // (nnz_pad) counts (acc_mode 0), padding 0
    std::vector<int64_t> pwfx;        // (nnz_pad) Q32.32 weights (acc_mode 1), padding 0
    int32_t max_chunks = 0;           // work items of the longest padded row
    int64_t chunks_all = 0;           // work items if every neuron fires (sum over padded rows)
    std::vector<int64_t> chunk_cum;   // (n+1) work items of rows 0..i-1
};

// Work items if every pair of one list segment fires, maximised over the segments: segment c holds
// the pairs [c * seg_pairs, (c+1) * seg_pairs) of a group of `group` instances (pair (b, i) =
// b * n_pad + i; pairs with i >= n are padding and never fire).
inline int64_t segment_capacity(const HostCsr& H, int64_t n_pad, int64_t group, int64_t seg_pairs, int64_t n_seg)
{
    auto upto = [&](int64_t p) {                  // items of the pairs [0, p)
        const int64_t b = p / n_pad, i = std::min(p - b * n_pad, H.n);
        return b * H.chunks_all + H.chunk_cum[i];
    };
    const int64_t pairs = group * n_pad;
    int64_t cap = 1;
    for (int64_t c = 0; c < n_seg; c++) {
        const int64_t lo = std::min(c * seg_pairs, pairs), hi = std::min(lo + seg_pairs, pairs);
        cap = std::max(cap, upto(hi) - upto(lo));
    }
    return cap;
}

// Returns "" on success or the error message.
inline std::string prepare_csr(const int64_t* indptr, const int32_t* indices, const float* data, int64_t n,
                               int64_t nnz, float w_syn32, bool force_fixed, HostCsr& H)
{
    char msg[256];
    H = HostCsr{};
    H.n = n;
    H.nnz = nnz;
    if (n <= 0 || nnz < 0) return "empty network";
    if (indptr[0] != 0 || indptr[n] != nnz) return "indptr must start at 0 and end at nnz";
    H.ip.assign(indptr, indptr + n + 1);
    H.ix.resize(nnz);
    std::vector<float> dv(nnz);
    std::vector<int64_t> perm;
    for (int64_t i = 0; i < n; i++) {
        const int64_t a = H.ip[i], b = H.ip[i + 1];
        if (b < a || b > nnz) {
            std::snprintf(msg, sizeof(msg), "indptr decreases at row %lld", (long long)i);
            return msg;
        }
        perm.resize(b - a);
        for (int64_t k = a; k < b; k++) perm[k - a] = k;
        std::stable_sort(perm.begin(), perm.end(), [&](int64_t x, int64_t y) { return indices[x] < indices[y]; });
        for (int64_t k = a; k < b; k++) {
            const int32_t c = indices[perm[k - a]];
            if (c < 0 || c >= n) {
                std::snprintf(msg, sizeof(msg), "column %d out of range in row %lld", c, (long long)i);
                return msg;
            }
            if (k > a && c == H.ix[k - 1]) {
                std::snprintf(msg, sizeof(msg), "duplicate column %d in row %lld", c, (long long)i);
                return msg;
            }
            H.ix[k] = c;
            dv[k] = data[perm[k - a]];
        }
    }
    bool integral = !force_fixed;
    for (int64_t k = 0; k < nnz && integral; k++)
        if (!(dv[k] == std::nearbyint(dv[k])) || std::fabs(dv[k]) > 32767.0f) integral = false;
    H.acc_mode = integral ? 0 : 1;
    H.wd.resize(nnz);
    for (int64_t k = 0; k < nnz; k++) H.wd[k] = dv[k] * w_syn32;

    H.rp.assign(n + 1, 0);
    H.chunk_cum.assign(n + 1, 0);
    int64_t max_pad = 0;
    for (int64_t i = 0; i < n; i++) {
        const int64_t len = H.ip[i + 1] - H.ip[i];
        const int64_t padded = (len + HOST_EDGE_ALIGN - 1) / HOST_EDGE_ALIGN * HOST_EDGE_ALIGN;
        H.rp[i + 1] = H.rp[i] + padded;
        max_pad = std::max(max_pad, padded);
        H.chunks_all += (padded + HOST_CHUNK - 1) / HOST_CHUNK;
        H.chunk_cum[i + 1] = H.chunks_all;
    }
    H.nnz_pad = H.rp[n];
    H.max_chunks = (int32_t)((max_pad + HOST_CHUNK - 1) / HOST_CHUNK);
    if (H.max_chunks >= (1 << HOST_CHUNK_BITS)) {
        std::snprintf(msg, sizeof(msg), "a row of %lld entries is too long", (long long)max_pad);
        return msg;
    }
    H.pcol.assign(H.nnz_pad, 0);
    if (H.acc_mode == 0) H.pcnt.assign(H.nnz_pad, 0);
    else H.pwfx.assign(H.nnz_pad, 0);
    for (int64_t i = 0; i < n; i++) {
        int64_t q = H.rp[i];
        for (int64_t k = H.ip[i]; k < H.ip[i + 1]; k++, q++) {
            H.pcol[q] = H.ix[k];
            if (H.acc_mode == 0) H.pcnt[q] = (int16_t)std::nearbyint(dv[k]);
            else H.pwfx[q] = q32_host(H.wd[k]);
        }
    }
    return "";
}

// The connectome by postsynaptic neuron (the pull propagation's gather order): for post j the
// entries colptr[j]..colptr[j+1]-1 hold (presynaptic neuron, count or Q32.32 weight), by pre.
struct HostCsc {
    std::vector<int64_t> colptr;      // (n+1)
    std::vector<int32_t> pre;         // (nnz)
    std::vector<int16_t> cnt;         // (nnz) acc_mode 0
    std::vector<int64_t> wfx;         // (nnz) acc_mode 1
};

inline void build_csc(const HostCsr& H, HostCsc& C)
{
    const int64_t n = H.n, nnz = H.nnz;
    C = HostCsc{};
    C.colptr.assign(n + 1, 0);
    for (int64_t k = 0; k < nnz; k++) C.colptr[H.ix[k] + 1] += 1;
    for (int64_t j = 0; j < n; j++) C.colptr[j + 1] += C.colptr[j];
    std::vector<int64_t> fill(C.colptr.begin(), C.colptr.end() - 1);
    C.pre.resize(nnz);
    if (H.acc_mode == 0) C.cnt.resize(nnz);
    else C.wfx.resize(nnz);
    for (int64_t i = 0; i < n; i++)
        for (int64_t k = H.ip[i]; k < H.ip[i + 1]; k++) {
            const int64_t q = fill[H.ix[k]]++;
            const int64_t src = H.rp[i] + (k - H.ip[i]);
            C.pre[q] = (int32_t)i;
            if (H.acc_mode == 0) C.cnt[q] = H.pcnt[src];
            else C.wfx[q] = H.pwfx[src];
        }
}

struct PlasticPlan {
    int64_t n_pl = 0;
    int32_t n_ppost = 0;
    std::vector<int64_t> pos;         // sorted, unique CSR positions
    std::vector<int64_t> plr;         // (n+1) plastic entries grouped by presynaptic neuron
    std::vector<int32_t> pl_pidx;     // (n_pl) compact target index
    std::vector<int64_t> q0;          // (n_pl) q32 of the connectome weight
    std::vector<float> w0;            // (n_pl) connectome weight f32(count * w_syn)
    std::vector<int32_t> ppost_of;    // (n) compact target index or -1
    std::vector<int32_t> pre;         // (n_pl) presynaptic neuron of each entry
    std::vector<int32_t> post;        // (n_pl) postsynaptic neuron of each entry
    std::vector<int32_t> ppost_neuron;// (n_ppost) neuron of each compact target
};

// Plan the plastic side for positions `pos` (any order, duplicates allowed). "" or an error.
inline std::string plan_plastic(const HostCsr& H, std::vector<int64_t> pos, PlasticPlan& P)
{
    P = PlasticPlan{};
    std::sort(pos.begin(), pos.end());
    pos.erase(std::unique(pos.begin(), pos.end()), pos.end());
    for (int64_t p : pos)
        if (p < 0 || p >= H.nnz) {
            char msg[128];
            std::snprintf(msg, sizeof(msg), "plastic position %lld out of range", (long long)p);
            return msg;
        }
    const int64_t n = H.n, n_pl = (int64_t)pos.size();
    P.n_pl = n_pl;
    P.pos = pos;
    P.plr.assign(n + 1, 0);
    P.ppost_of.assign(n, -1);
    P.pl_pidx.resize(n_pl);
    P.q0.resize(n_pl);
    P.w0.resize(n_pl);
    std::vector<int32_t> up;
    up.reserve(n_pl);
    for (int64_t k = 0; k < n_pl; k++) up.push_back(H.ix[pos[k]]);
    std::sort(up.begin(), up.end());
    up.erase(std::unique(up.begin(), up.end()), up.end());
    for (size_t q = 0; q < up.size(); q++) P.ppost_of[up[q]] = (int32_t)q;
    P.n_ppost = (int32_t)up.size();
    P.ppost_neuron = up;
    P.pre.resize(n_pl);
    P.post.resize(n_pl);
    int64_t r = 0;
    for (int64_t k = 0; k < n_pl; k++) {
        while (H.ip[r + 1] <= pos[k]) r++;          // row containing position pos[k]
        P.pre[k] = (int32_t)r;
        P.post[k] = H.ix[pos[k]];
        P.pl_pidx[k] = P.ppost_of[H.ix[pos[k]]];
        P.w0[k] = H.wd[pos[k]];
        P.q0[k] = q32_host(P.w0[k]);
        P.plr[r + 1] += 1;
    }
    for (int64_t i = 0; i < n; i++) P.plr[i + 1] += P.plr[i];
    return "";
}

// Per-instance weights for a new plan: entries plastic before keep their (B, old) values.
inline std::vector<float> remap_weights(const PlasticPlan& old_plan, const std::vector<float>& old_pw,
                                        const PlasticPlan& P, int32_t B)
{
    std::vector<float> pw((size_t)B * P.n_pl);
    for (int32_t b = 0; b < B; b++) std::copy(P.w0.begin(), P.w0.end(), pw.begin() + (size_t)b * P.n_pl);
    for (int64_t k = 0, j = 0; k < old_plan.n_pl; k++) {
        while (j < P.n_pl && P.pos[j] < old_plan.pos[k]) j++;
        if (j < P.n_pl && P.pos[j] == old_plan.pos[k])
            for (int32_t b = 0; b < B; b++) pw[(size_t)b * P.n_pl + j] = old_pw[(size_t)b * old_plan.n_pl + k];
    }
    return pw;
}

// Plastic input in flight, (R*B, old n_ppost) -> (R*B, new n_ppost), renumbered by target neuron.
inline std::vector<int64_t> remap_ring(const PlasticPlan& old_plan, const std::vector<int64_t>& old_ring,
                                       const PlasticPlan& P, int64_t rows)
{
    std::vector<int64_t> ring((size_t)rows * std::max(1, P.n_ppost), 0);
    if (old_plan.n_ppost == 0) return ring;
    std::vector<int32_t> old_post(old_plan.n_ppost, -1);
    for (int64_t i = 0; i < (int64_t)old_plan.ppost_of.size(); i++)
        if (old_plan.ppost_of[i] >= 0) old_post[old_plan.ppost_of[i]] = (int32_t)i;
    for (int64_t r = 0; r < rows; r++)
        for (int32_t q = 0; q < old_plan.n_ppost; q++) {
            const int64_t x = old_ring[(size_t)r * old_plan.n_ppost + q];
            if (x) ring[(size_t)r * P.n_ppost + P.ppost_of[old_post[q]]] = x;
        }
    return ring;
}

}  // namespace fb
