// C ABI of the B200 LIF engine (include/flybrain.h): host orchestration of the kernels in
// engine.cuh (step engine) and persist.cuh (persistent engine).
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "../../include/flybrain.h"
#include "engine.cuh"
#include "host_prep.hpp"
#include "persist.cuh"
#include "plastic.cuh"
#include "readout.cuh"
#include "instruct.cuh"
#include "eye.cuh"

using namespace fb;

namespace {

thread_local std::string g_err;

}  // namespace

namespace fb {
void set_last_error(const char* msg) { g_err = msg; }
}  // namespace fb

namespace {

int fail(int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CU(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) return fail(FB_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

template <typename T> int dalloc(T** p, size_t count, size_t* total)
{
    *p = nullptr;
    size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    CU(cudaMalloc((void**)p, bytes));
    *total += bytes;
    return FB_OK;
}

template <typename T> int upload(T** p, const std::vector<T>& h, size_t* total)
{
    int rc = dalloc(p, h.size(), total);
    if (rc) return rc;
    if (!h.empty()) CU(cudaMemcpy(*p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    return FB_OK;
}

// FP64 constants computed on the device (exp(-dt/tau) in double), then rounded for FP32 state.
__global__ void k_consts(double dt, double tau_m, double tau_syn, double f_poisson, double w_syn, double* out)
{
    out[0] = exp(-dt / tau_syn);
    out[1] = dt / tau_m;
    out[2] = f_poisson * w_syn;
}

template <typename Real>
__global__ void k_reset(Real* v, Real* g, int8_t* ref, void* acc, int32_t n_slots, int acc_bytes, int64_t* pring,
                        int32_t R, int32_t B, int64_t n, int64_t n_pad, int32_t n_ppost, const uint8_t* fly_mask,
                        Real v_rest)
{
    const int64_t total = (int64_t)B * n;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < total; p += stride) {
        const int32_t b = (int32_t)(p / n);
        if (fly_mask && !fly_mask[b]) continue;
        v[p] = v_rest;
        g[p] = (Real)0;
        ref[p] = 0;
        const int64_t a = (int64_t)b * n_pad + (p - (int64_t)b * n);
        for (int32_t k = 0; k < n_slots; k++) {
            const int64_t o = (int64_t)k * B * n_pad + a;
            if (acc_bytes == 4) ((int32_t*)acc)[o] = 0;
            else ((int64_t*)acc)[o] = 0;
        }
    }
    const int64_t ptotal = (int64_t)R * B * n_ppost;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < ptotal; p += stride) {
        const int32_t b = (int32_t)((p / n_ppost) % B);
        if (fly_mask && !fly_mask[b]) continue;
        pring[p] = 0;
    }
}

__global__ void k_set_ticks(int64_t* reset_tick, const uint8_t* fly_mask, int32_t B, int64_t t)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < B && (!fly_mask || fly_mask[b])) reset_tick[b] = t;
}

}  // namespace

struct fb_brain {
    int device = 0;
    fb_params params{};
    int64_t n = 0, n_pad = 0, nnz = 0, nnz_pad = 0;
    int32_t B = 0, n_delay = 1, n_ref = 0, R = 2, R_pl = 2;
    int acc_mode = 0;      // 0 INT32 counts, 1 Q32.32
    int f64 = 0;
    uint32_t seed = 0;
    double consts64[3] = {0, 0, 0};
    Lif<float> L32{};
    Lif<double> L64{};
    // connectome
    int64_t* rowptr = nullptr;
    int32_t* col = nullptr;
    int16_t* cnt = nullptr;
    int64_t* wfx = nullptr;
    int32_t max_chunks = 0;
    // plastic
    int64_t n_pl = 0;
    int32_t pl_mode = 0;              // 0 no plastic synapses, 1 plastic, 2 plastic in long rows
    int32_t n_ppost = 0;
    int64_t* pl_rowptr = nullptr;
    int32_t* pl_pidx = nullptr;
    int64_t* pl_q0 = nullptr;
    int32_t* pl_pre = nullptr;        // presynaptic / postsynaptic neuron of each plastic entry
    int32_t* pl_post = nullptr;
    int32_t* ppost_neuron = nullptr;  // neuron of each compact plastic target
    int32_t* ppost_of = nullptr;
    // pull propagation (built on first use): connectome by postsynaptic neuron + spike masks
    int64_t* colptr = nullptr;
    int32_t* cpre = nullptr;
    int16_t* ccnt = nullptr;
    int64_t* cwfx = nullptr;
    unsigned long long* masks = nullptr;
    int32_t mask_words = 0;
    int64_t mask_from = 0;        // first spike step whose mask is recorded (pull reads only these)
    bool masks_dirty = false;     // steps ran without recording masks (the persistent engine)
    float* pw = nullptr;
    float* w0 = nullptr;
    // state
    void* v = nullptr;
    void* g = nullptr;
    int8_t* ref = nullptr;
    // ext
    std::vector<int32_t> h_ext_idx;
    int32_t* ext_idx = nullptr;
    int64_t n_ext = 0;
    float* p_ext = nullptr;
    float* bias_ext = nullptr;
    std::vector<void*> graveyard;     // superseded buffers, freed at destroy (callers may hold views)
    HostCsr hc;                       // host copy of the CSR for re-planning the plastic entries
    PlasticPlan plastic;              // current plastic plan
    // delay line
    void* acc = nullptr;          // [n_slots][B][n_pad]
    int32_t n_slots = 2;
    int32_t epoch = 1;            // persistent engine: steps per grid barrier
    int64_t pushed_until = 1;     // the arrivals of every tick < pushed_until are in acc
    int64_t* pring = nullptr;
    int2* items = nullptr;
    int32_t* item_count = nullptr;
    int64_t cap_c = 0;            // items per (step, group, segment) list (<= cap_alloc)
    int64_t cap_alloc = 0;        // ... as allocated
    long long barrier_cycles = BARRIER_TIMEOUT_CYCLES;   // persistent engine's grid-barrier wait budget
    int32_t list_group = 1;       // instances per group (the persistent group size, or B)
    int32_t n_groups = 1;
    int32_t n_seg = 1;            // segments per group (the persistent CTAs, or 1)
    int64_t seg_pairs = 0;        // pairs per segment
    unsigned int* bar = nullptr;  // persistent grid-barrier counter
    int32_t* abort_flag = nullptr;
    int2* ext_tab = nullptr;      // persistent engine: input pairs of each CTA
    int32_t* ext_off = nullptr;
    int64_t* reset_tick = nullptr;
    int64_t* stop_tick = nullptr;
    uint8_t* fly_mask = nullptr;
    // pinned staging of fb_reset's instance masks: a ring of buffers, each reused only after the
    // copy that read it completed (its event), so a partial reset never blocks on the stream
    static constexpr int MASK_RING = 4;
    uint8_t* mask_h[MASK_RING] = {nullptr};
    cudaEvent_t mask_ev[MASK_RING] = {nullptr};
    bool mask_used[MASK_RING] = {false};
    int mask_at = 0;
    long long* trace = nullptr;   // caller's phase-trace buffer (fb_set_trace) or nullptr
    int64_t trace_cap = 0;
    int32_t* err_h = nullptr;   // host-mapped flags
    int32_t* err_d = nullptr;
    // counters
    int64_t t = 0;
    uint32_t step_no = 0;
    int64_t launches = 0;
    size_t bytes = 0;
    // schedule
    int engine = FB_ENGINE_AUTO;
    int prop = FB_PROP_PUSH;
    int lanes = 8;
    int sm_count = 148;
    PersistPlan plan{};

    DevNet net() const
    {
        DevNet N{};
        N.n = n; N.n_pad = n_pad; N.B = B; N.n_delay = n_delay; N.R = R; N.R_pl = R_pl; N.n_ref = n_ref;
        N.rowptr = rowptr; N.col = col; N.cnt = cnt; N.wfx = wfx;
        N.n_pl = n_pl; N.n_ppost = n_ppost; N.pl_rowptr = pl_rowptr; N.pl_pidx = pl_pidx; N.pl_q0 = pl_q0;
        N.ppost_of = ppost_of;
        N.colptr = colptr; N.cpre = cpre; N.ccnt = ccnt; N.cwfx = cwfx;
        N.L32 = L32; N.L64 = L64;
        return N;
    }
    DevState state() const
    {
        DevState S{};
        S.v = v; S.g = g; S.ref = ref; S.pw = pw; S.ext_idx = ext_idx; S.n_ext = (int32_t)n_ext;
        S.p_ext = p_ext; S.bias_ext = bias_ext; S.acc = acc; S.n_slots = n_slots; S.pring = pring;
        S.items = items; S.item_count = item_count; S.cap_c = cap_c; S.group = list_group;
        S.n_groups = n_groups; S.n_seg = n_seg; S.seg_pairs = seg_pairs; S.reset_tick = reset_tick;
        S.stop_tick = stop_tick; S.err = err_d; S.seed = seed;
        S.masks = masks; S.mask_words = mask_words;
        return S;
    }
};

namespace {

int free_all(fb_brain* h)
{
    void* ptrs[] = {h->rowptr, h->col, h->cnt, h->wfx, h->pl_rowptr, h->pl_pidx, h->pl_q0, h->ppost_of, h->pw, h->w0,
                    h->pl_pre, h->pl_post, h->ppost_neuron,
                    h->v, h->g, h->ref, h->ext_idx, h->p_ext, h->bias_ext, h->acc, h->pring,
                    h->items, h->item_count, h->reset_tick, h->stop_tick, h->fly_mask, h->bar, h->abort_flag,
                    h->ext_tab, h->ext_off, h->colptr, h->cpre, h->ccnt, h->cwfx, h->masks};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    for (void* p : h->graveyard) cudaFree(p);
    if (h->err_h) cudaFreeHost(h->err_h);
    for (int k = 0; k < fb_brain::MASK_RING; k++) {
        if (h->mask_ev[k]) cudaEventDestroy(h->mask_ev[k]);
        if (h->mask_h[k]) cudaFreeHost(h->mask_h[k]);
    }
    return FB_OK;
}

int64_t py_round(double x) { return (int64_t)std::nearbyint(x); }   // round half to even, like Python

// (Re)build the plastic side for CSR positions `pos`. Per-instance weights of positions that
// were plastic before are kept, new ones start at the connectome weight; plastic input in flight
// is carried over to the new compact target numbering. The device must be idle.
int install_plastic(fb_brain* h, const std::vector<int64_t>& pos)
{
    PlasticPlan P;
    std::string err = plan_plastic(h->hc, pos, P);
    if (!err.empty()) return fail(FB_ERR_ARG, "%s", err.c_str());
    const int32_t B = h->B;
    std::vector<float> old_pw((size_t)B * h->n_pl);
    if (h->n_pl > 0) CU(cudaMemcpy(old_pw.data(), h->pw, old_pw.size() * sizeof(float), cudaMemcpyDeviceToHost));
    std::vector<float> pwh = remap_weights(h->plastic, old_pw, P, B);
    std::vector<int64_t> old_ring;
    if (h->pring && h->n_ppost > 0) {
        old_ring.resize((size_t)h->R_pl * B * h->n_ppost);
        CU(cudaMemcpy(old_ring.data(), h->pring, old_ring.size() * sizeof(int64_t), cudaMemcpyDeviceToHost));
    }
    std::vector<int64_t> ring = remap_ring(h->plastic, old_ring, P, (int64_t)h->R_pl * B);
    void* olds[] = {h->pl_rowptr, h->pl_pidx, h->pl_q0, h->ppost_of, h->w0, h->pring, h->pl_pre, h->pl_post,
                    h->ppost_neuron};
    for (void* p : olds)
        if (p) cudaFree(p);
    if (h->pw) h->graveyard.push_back(h->pw);   // callers may still hold a view of the old weights
    h->pl_rowptr = nullptr; h->pl_pidx = nullptr; h->pl_q0 = nullptr; h->ppost_of = nullptr;
    h->w0 = nullptr; h->pring = nullptr; h->pw = nullptr;
    h->pl_pre = nullptr; h->pl_post = nullptr; h->ppost_neuron = nullptr;
    size_t* tb = &h->bytes;
    int rc;
    if ((rc = upload(&h->pl_pre, P.pre, tb))) return rc;
    if ((rc = upload(&h->pl_post, P.post, tb))) return rc;
    if ((rc = upload(&h->ppost_neuron, P.ppost_neuron, tb))) return rc;
    if ((rc = upload(&h->pl_rowptr, P.plr, tb))) return rc;
    if ((rc = upload(&h->pl_pidx, P.pl_pidx, tb))) return rc;
    if ((rc = upload(&h->pl_q0, P.q0, tb))) return rc;
    if ((rc = upload(&h->ppost_of, P.ppost_of, tb))) return rc;
    if ((rc = upload(&h->w0, P.w0, tb))) return rc;
    if ((rc = upload(&h->pw, pwh, tb))) return rc;
    if ((rc = upload(&h->pring, ring, tb))) return rc;
    h->n_pl = P.n_pl;
    h->n_ppost = P.n_ppost;
    {   // long plastic rows (on average two or more plastic synapses per presynaptic neuron with any):
        // the persistent engine batches their pushes
        int64_t rows = 0;
        for (size_t r = 0; r + 1 < P.plr.size(); r++) rows += P.plr[r + 1] > P.plr[r];
        h->pl_mode = P.n_pl == 0 ? 0 : (P.n_pl >= 2 * std::max<int64_t>(rows, 1) ? 2 : 1);
    }
    h->plastic = std::move(P);
    return FB_OK;
}

// Per-CTA table of the persistent engine's input pairs (pairs whose neuron has an ext slot):
// entry {local pair | instance-in-group << 18, ext slot}, grouped by CTA. Rebuilt when the ext
// map changes; the same table serves every group (pairs are numbered within a group).
int build_ext_table(fb_brain* h)
{
    const PersistPlan& P = h->plan;
    if (P.group == 0) return FB_OK;
    std::vector<int32_t> off(P.ctas + 1, 0);
    std::vector<int2> tab;
    const int64_t np = h->n_pad, total = (int64_t)P.group * np;
    for (int32_t c = 0; c < P.ctas; c++) {
        off[c] = (int32_t)tab.size();
        const int64_t lo = (int64_t)c * P.per, hi = std::min(lo + P.per, total);
        for (int64_t p = lo; p < hi; p++) {
            const int64_t bl = p / np, i = p - bl * np;
            if (i < h->n && h->h_ext_idx[i] >= 0) tab.push_back(make_int2((int32_t)((p - lo) | (bl << 18)), h->h_ext_idx[i]));
        }
    }
    off[P.ctas] = (int32_t)tab.size();
    if (h->ext_tab) h->graveyard.push_back(h->ext_tab);
    if (h->ext_off) h->graveyard.push_back(h->ext_off);
    h->ext_tab = nullptr;
    h->ext_off = nullptr;
    int rc = upload(&h->ext_tab, tab, &h->bytes);
    if (rc) return rc;
    return upload(&h->ext_off, off, &h->bytes);
}

int dispatch_step(fb_brain* h, const StepArgs& A, bool raster, bool record, cudaStream_t st);
int dispatch_push(fb_brain* h, int64_t t, cudaStream_t st);
int dispatch_pull(fb_brain* h, int64_t t, cudaStream_t st);

// Build what pull propagation needs: the connectome by postsynaptic neuron and the spike-mask
// ring (zeroed; masks are recorded from the current step on). The device must be idle.
int enable_pull(fb_brain* h)
{
    if (h->masks) return FB_OK;
    HostCsc Cc;
    build_csc(h->hc, Cc);
    int rc;
    if ((rc = upload(&h->colptr, Cc.colptr, &h->bytes))) return rc;
    if ((rc = upload(&h->cpre, Cc.pre, &h->bytes))) return rc;
    if (h->acc_mode == 0) { if ((rc = upload(&h->ccnt, Cc.cnt, &h->bytes))) return rc; }
    else if ((rc = upload(&h->cwfx, Cc.wfx, &h->bytes))) return rc;
    h->mask_words = (h->B + 63) / 64;
    const size_t words = (size_t)h->R * h->n * h->mask_words;
    if ((rc = dalloc(&h->masks, words, &h->bytes))) return rc;
    CU(cudaMemset(h->masks, 0, words * sizeof(unsigned long long)));
    h->mask_from = h->t;
    h->masks_dirty = false;
    return FB_OK;
}

}  // namespace

extern "C" int fb_last_error(char* buf, int64_t len)
{
    if (!buf || len <= 0) return FB_ERR_ARG;
    std::snprintf(buf, (size_t)len, "%s", g_err.c_str());
    return FB_OK;
}

extern "C" int fb_create(const fb_params* P, const int64_t* indptr, const int32_t* indices, const float* data,
                         int64_t n, int64_t nnz, int32_t batch, uint32_t seed, const int64_t* plastic_pos,
                         int64_t n_plastic, uint32_t flags, int32_t device, fb_brain** out)
{
    if (!out) return fail(FB_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (!P || n <= 0 || nnz < 0 || batch <= 0 || !indptr || (nnz > 0 && (!indices || !data)))
        return fail(FB_ERR_ARG, "bad connectome arguments (n=%lld nnz=%lld batch=%d)", (long long)n, (long long)nnz, batch);
    if (n > (int64_t)INT32_MAX - 1) return fail(FB_ERR_ARG, "n=%lld exceeds the int32 neuron index", (long long)n);
    if (batch >= (1 << (31 - CHUNK_BITS))) return fail(FB_ERR_ARG, "batch %d too large", batch);
    if (P->dt <= 0 || P->tau_m <= 0 || P->tau_syn <= 0) return fail(FB_ERR_ARG, "dt, tau_m, tau_syn must be > 0");
    CU(cudaSetDevice(device));
    fb_brain* h = new fb_brain();
    h->device = device;
    h->params = *P;
    h->n = n;
    h->nnz = nnz;
    h->B = batch;
    h->seed = seed;
    h->f64 = (flags & FB_FLAG_F64) ? 1 : 0;
    h->n_delay = (int32_t)std::max<int64_t>(1, py_round(P->delay / P->dt));
    h->n_ref = (int32_t)py_round(P->t_ref / P->dt);
    h->R = h->n_delay + 1;
    h->n_pad = (n + 15) / 16 * 16;
    if (h->n_ref < 0 || h->n_ref > 127) { delete h; return fail(FB_ERR_ARG, "n_ref=%d must fit int8", h->n_ref); }
    int dev_sms = 0;
    cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, device);
    h->sm_count = dev_sms > 0 ? dev_sms : 148;

    // --- host CSR: validate, sort columns within rows, classify weights, pad rows ------------
    {
        std::string err = prepare_csr(indptr, indices, data, n, nnz, (float)P->w_syn,
                                      (flags & FB_FLAG_ACC_FIXED) != 0, h->hc);
        if (!err.empty()) { delete h; return fail(FB_ERR_ARG, "%s", err.c_str()); }
    }
    const HostCsr& H = h->hc;
    h->acc_mode = H.acc_mode;
    h->nnz_pad = H.nnz_pad;
    h->max_chunks = H.max_chunks;
    std::vector<int64_t> pos(plastic_pos, plastic_pos + std::max<int64_t>(0, n_plastic));

    // --- device allocations -------------------------------------------------------------------
    int rc = FB_OK;
    size_t* tb = &h->bytes;
#define TRY(x) do { rc = (x); if (rc) { free_all(h); delete h; return rc; } } while (0)
    TRY(upload(&h->rowptr, H.rp, tb));
    TRY(upload(&h->col, H.pcol, tb));
    if (h->acc_mode == 0) TRY(upload(&h->cnt, H.pcnt, tb));
    else TRY(upload(&h->wfx, H.pwfx, tb));
    const size_t nb = (size_t)batch * n;
    const size_t rs = h->f64 ? sizeof(double) : sizeof(float);
    TRY(dalloc((char**)&h->v, nb * rs, tb));
    TRY(dalloc((char**)&h->g, nb * rs, tb));
    TRY(dalloc(&h->ref, nb, tb));
    h->h_ext_idx.assign(n, -1);
    TRY(upload(&h->ext_idx, h->h_ext_idx, tb));
    TRY(dalloc(&h->p_ext, 1, tb));
    TRY(dalloc(&h->bias_ext, 1, tb));
    const size_t ab = h->acc_mode == 0 ? 4 : 8;
    const size_t nbp = (size_t)batch * h->n_pad;
    TRY(dalloc(&h->bar, 1, tb));
    TRY(dalloc(&h->abort_flag, 1, tb));
    int dev_sms2 = h->sm_count;
    h->plan = plan_persistent(h->n, h->n_pad, h->B, h->f64 != 0, h->n_ref, h->n_delay, (int)ab, dev_sms2, h->device);
    // the persistent engine runs epochs of K steps between grid barriers: the spikes of an epoch
    // arrive two epochs later at the earliest when 2K + 1 <= n_delay; 2K accumulator slots
    h->epoch = h->plan.group > 0 ? std::max(1, std::min(MAX_EPOCH, (h->n_delay - 1) / 2)) : 1;
    h->n_slots = 2 * h->epoch;
    h->R_pl = h->n_delay + h->epoch;
    TRY(dalloc((char**)&h->acc, nbp * ab * h->n_slots, tb));
    CU(cudaMemset(h->acc, 0, nbp * ab * h->n_slots));
    h->list_group = h->plan.group > 0 ? h->plan.group : h->B;
    h->n_groups = (h->B + h->list_group - 1) / h->list_group;
    TRY(install_plastic(h, pos));
    TRY(build_ext_table(h));
    // one list segment per persistent CTA (the pairs it owns); capacity for the worst case, every
    // pair of the segment firing in the same step
    h->n_seg = h->plan.group > 0 ? h->plan.ctas : 1;
    h->seg_pairs = h->plan.group > 0 ? h->plan.per : (int64_t)h->list_group * h->n_pad;
    h->cap_c = segment_capacity(H, h->n_pad, h->list_group, h->seg_pairs, h->n_seg);
    h->cap_alloc = h->cap_c;
    TRY(dalloc(&h->items, (size_t)h->R * h->n_groups * h->n_seg * h->cap_c, tb));
    TRY(dalloc(&h->item_count, (size_t)h->R * h->n_groups * h->n_seg, tb));
    TRY(dalloc(&h->reset_tick, (size_t)batch, tb));
    TRY(dalloc(&h->stop_tick, (size_t)batch, tb));
    TRY(dalloc(&h->fly_mask, (size_t)batch, tb));
    {
        std::vector<int64_t> st(batch, std::numeric_limits<int64_t>::max());
        CU(cudaMemcpy(h->stop_tick, st.data(), batch * sizeof(int64_t), cudaMemcpyHostToDevice));
    }
    CU(cudaHostAlloc((void**)&h->err_h, 4 * sizeof(int32_t), cudaHostAllocMapped));
    std::memset(h->err_h, 0, 4 * sizeof(int32_t));
    CU(cudaHostGetDevicePointer((void**)&h->err_d, h->err_h, 0));

    // FP64 decay factors on the device
    {
        double* d = nullptr;
        CU(cudaMalloc(&d, 3 * sizeof(double)));
        k_consts<<<1, 1>>>(P->dt, P->tau_m, P->tau_syn, P->f_poisson, P->w_syn, d);
        CU(cudaGetLastError());
        CU(cudaMemcpy(h->consts64, d, 3 * sizeof(double), cudaMemcpyDeviceToHost));
        cudaFree(d);
        h->launches += 1;
    }
    h->L32 = Lif<float>{(float)h->consts64[0], (float)h->consts64[1], (float)h->consts64[2], (float)P->w_syn,
                        (float)P->v_rest, (float)P->v_th, (float)P->v_reset};
    h->L64 = Lif<double>{h->consts64[0], h->consts64[1], h->consts64[2], P->w_syn, P->v_rest, P->v_th, P->v_reset};
    rc = fb_reset(h, nullptr, -1, nullptr);
    if (rc) { free_all(h); delete h; return rc; }
    CU(cudaDeviceSynchronize());
#undef TRY
    *out = h;
    return FB_OK;
}

extern "C" int fb_destroy(fb_brain* h)
{
    if (!h) return FB_OK;
    cudaSetDevice(h->device);
    cudaDeviceSynchronize();
    free_all(h);
    delete h;
    return FB_OK;
}

extern "C" int fb_get_info(const fb_brain* h, fb_info* o)
{
    if (!h || !o) return fail(FB_ERR_ARG, "NULL argument");
    std::memset(o, 0, sizeof(*o));
    o->n = h->n; o->nnz = h->nnz; o->batch = h->B; o->n_delay = h->n_delay; o->n_ref = h->n_ref;
    o->acc_mode = h->acc_mode; o->f64 = h->f64; o->engine = h->engine; o->propagation = h->prop;
    o->lanes = h->lanes; o->group = h->plan.group; o->ctas = h->plan.ctas; o->n_plastic = h->n_pl;
    o->n_ext = h->n_ext; o->t = h->t; o->step_no = h->step_no; o->launches = h->launches;
    o->item_capacity = h->cap_c; o->bytes_device = (int64_t)h->bytes; o->epoch = h->epoch;
    o->decay_syn = h->consts64[0]; o->decay_m = h->consts64[1]; o->kick = h->consts64[2];
    return FB_OK;
}

extern "C" int fb_get_views(fb_brain* h, fb_views* o)
{
    if (!h || !o) return fail(FB_ERR_ARG, "NULL argument");
    o->v = h->v; o->g = h->g; o->ref = h->ref; o->pw = h->pw; o->w0 = h->w0; o->ext_idx = h->ext_idx;
    o->p_ext = h->p_ext; o->bias_ext = h->bias_ext; o->stop_tick = h->stop_tick;
    return FB_OK;
}

extern "C" int fb_set_ext(fb_brain* h, const int64_t* idx, int64_t count)
{
    if (!h || (count > 0 && !idx)) return fail(FB_ERR_ARG, "NULL argument");
    CU(cudaSetDevice(h->device));
    std::vector<int64_t> fresh;
    for (int64_t k = 0; k < count; k++) {
        if (idx[k] < 0 || idx[k] >= h->n) return fail(FB_ERR_ARG, "neuron %lld out of range", (long long)idx[k]);
        if (h->h_ext_idx[idx[k]] < 0) fresh.push_back(idx[k]);
    }
    std::sort(fresh.begin(), fresh.end());
    fresh.erase(std::unique(fresh.begin(), fresh.end()), fresh.end());
    if (fresh.empty()) return FB_OK;
    const int64_t old = h->n_ext, now = old + (int64_t)fresh.size();
    for (size_t k = 0; k < fresh.size(); k++) h->h_ext_idx[fresh[k]] = (int32_t)(old + (int64_t)k);
    CU(cudaDeviceSynchronize());
    CU(cudaMemcpy(h->ext_idx, h->h_ext_idx.data(), h->n * sizeof(int32_t), cudaMemcpyHostToDevice));
    float* np_ = nullptr;
    float* nb_ = nullptr;
    int rc = dalloc(&np_, (size_t)h->B * now, &h->bytes);
    if (rc) return rc;
    rc = dalloc(&nb_, (size_t)h->B * now, &h->bytes);
    if (rc) return rc;
    CU(cudaMemset(np_, 0, (size_t)h->B * now * sizeof(float)));
    CU(cudaMemset(nb_, 0, (size_t)h->B * now * sizeof(float)));
    if (old > 0) {
        CU(cudaMemcpy2D(np_, now * sizeof(float), h->p_ext, old * sizeof(float), old * sizeof(float), h->B, cudaMemcpyDeviceToDevice));
        CU(cudaMemcpy2D(nb_, now * sizeof(float), h->bias_ext, old * sizeof(float), old * sizeof(float), h->B, cudaMemcpyDeviceToDevice));
    }
    h->graveyard.push_back(h->p_ext);
    h->graveyard.push_back(h->bias_ext);
    h->p_ext = np_;
    h->bias_ext = nb_;
    h->n_ext = now;
    rc = build_ext_table(h);
    if (rc) return rc;
    CU(cudaDeviceSynchronize());
    return FB_OK;
}

extern "C" int fb_reset(fb_brain* h, const int32_t* flies, int32_t n_flies, void* stream)
{
    if (!h) return fail(FB_ERR_ARG, "NULL brain");
    CU(cudaSetDevice(h->device));
    cudaStream_t st = (cudaStream_t)stream;
    const bool all = (flies == nullptr || n_flies < 0);
    const uint8_t* mask = nullptr;
    if (!all) {
        for (int32_t k = 0; k < n_flies; k++)
            if (flies[k] < 0 || flies[k] >= h->B) return fail(FB_ERR_ARG, "fly %d out of range", flies[k]);
        const int r = h->mask_at;
        h->mask_at = (r + 1) % fb_brain::MASK_RING;
        if (!h->mask_h[r]) {
            CU(cudaHostAlloc((void**)&h->mask_h[r], (size_t)h->B, cudaHostAllocDefault));
            CU(cudaEventCreateWithFlags(&h->mask_ev[r], cudaEventDisableTiming));
        }
        if (h->mask_used[r]) CU(cudaEventSynchronize(h->mask_ev[r]));   // its last copy has been read
        std::memset(h->mask_h[r], 0, (size_t)h->B);
        for (int32_t k = 0; k < n_flies; k++) h->mask_h[r][flies[k]] = 1;
        CU(cudaMemcpyAsync(h->fly_mask, h->mask_h[r], h->B, cudaMemcpyHostToDevice, st));
        CU(cudaEventRecord(h->mask_ev[r], st));
        h->mask_used[r] = true;
        mask = h->fly_mask;
    }
    const int64_t total = (int64_t)h->B * h->n;
    const int blocks = (int)std::min<int64_t>((total + 255) / 256, (int64_t)h->sm_count * 16);
    const int ab = h->acc_mode == 0 ? 4 : 8;
    if (h->f64)
        k_reset<double><<<blocks, 256, 0, st>>>((double*)h->v, (double*)h->g, h->ref, h->acc, h->n_slots, ab, h->pring,
                                                h->R_pl, h->B, h->n, h->n_pad, h->n_ppost, mask, h->params.v_rest);
    else
        k_reset<float><<<blocks, 256, 0, st>>>((float*)h->v, (float*)h->g, h->ref, h->acc, h->n_slots, ab, h->pring,
                                               h->R_pl, h->B, h->n, h->n_pad, h->n_ppost, mask, (float)h->params.v_rest);
    CU(cudaGetLastError());
    h->launches += 1;
    if (all) {
        h->t = 0;
        h->pushed_until = 1;          // tick 0 receives nothing; nothing later is pushed
        if (h->masks) {
            CU(cudaMemsetAsync(h->masks, 0, (size_t)h->R * h->n * h->mask_words * sizeof(unsigned long long), st));
            h->mask_from = 0;
            h->masks_dirty = false;
        }
        CU(cudaMemsetAsync(h->item_count, 0, (size_t)h->R * h->n_groups * h->n_seg * sizeof(int32_t), st));
    }
    k_set_ticks<<<(h->B + 255) / 256, 256, 0, st>>>(h->reset_tick, mask, h->B, h->t);
    CU(cudaGetLastError());
    h->launches += 1;
    return FB_OK;
}

extern "C" int fb_set_plastic(fb_brain* h, const int64_t* pos, int64_t count)
{
    if (!h || (count > 0 && !pos)) return fail(FB_ERR_ARG, "NULL argument");
    CU(cudaSetDevice(h->device));
    std::vector<int64_t> all = h->plastic.pos;
    for (int64_t k = 0; k < count; k++) {
        if (pos[k] < 0 || pos[k] >= h->nnz) return fail(FB_ERR_ARG, "plastic position %lld out of range", (long long)pos[k]);
        all.push_back(pos[k]);
    }
    std::sort(all.begin(), all.end());
    all.erase(std::unique(all.begin(), all.end()), all.end());
    if (all.size() == h->plastic.pos.size()) return FB_OK;
    CU(cudaDeviceSynchronize());
    int rc = install_plastic(h, all);
    if (rc) return rc;
    CU(cudaDeviceSynchronize());
    return FB_OK;
}

extern "C" int fb_reward_step(fb_brain* h, const int32_t* counts, double* elig, float* post_mean, const double* coef,
                              const int32_t* fly_ptr, const int32_t* fly_slots, const float* fly_weight, int32_t n_flies,
                              const uint8_t* mask, double ae, double ap, float cap, int32_t apply, void* stream)
{
    if (!h || !counts || !elig || !post_mean) return fail(FB_ERR_ARG, "NULL argument");
    if (apply && (!coef || !fly_ptr || !fly_slots || !fly_weight || n_flies <= 0))
        return fail(FB_ERR_ARG, "apply needs coef, fly_ptr, fly_slots, fly_weight and n_flies > 0");
    if (h->n_pl == 0) return FB_OK;
    CU(cudaSetDevice(h->device));
    cudaStream_t st = (cudaStream_t)stream;
    RewardArgs a{};
    a.B = h->B; a.n_flies = n_flies; a.n = h->n; a.n_pl = h->n_pl; a.n_ppost = h->n_ppost;
    a.counts = counts; a.pre = h->pl_pre; a.post = h->pl_post; a.pidx = h->pl_pidx; a.ppost_neuron = h->ppost_neuron;
    a.w0 = h->w0; a.pw = h->pw; a.elig = elig; a.post_mean = post_mean; a.coef = coef;
    a.fly_ptr = fly_ptr; a.fly_slots = fly_slots; a.fly_weight = fly_weight; a.mask = mask;
    a.ae = ae; a.ap = ap; a.cap = cap; a.w_syn = (float)h->params.w_syn; a.apply = apply;
    k_reward_elig<<<(unsigned)(((int64_t)h->B * h->n_pl + 255) / 256), 256, 0, st>>>(a);
    CU(cudaGetLastError());
    if (apply) {
        k_reward_apply<<<(unsigned)(((int64_t)n_flies * h->n_pl + 255) / 256), 256, 0, st>>>(a);
        CU(cudaGetLastError());
        h->launches += 1;
    }
    const int64_t np_ = (int64_t)h->B * h->n_ppost;
    k_reward_post_mean<<<(unsigned)((np_ + 255) / 256), 256, 0, st>>>(a);
    CU(cudaGetLastError());
    h->launches += 2;
    return FB_OK;
}

extern "C" int fb_group_rates(const fb_brain* h, const int32_t* counts, const int32_t* idx, const int32_t* grp_ptr,
                              int32_t n_groups, const float* w, float a, float hz, float* rates, void* stream)
{
    if (!h || !counts || !idx || !grp_ptr || !w || !rates || n_groups <= 0) return fail(FB_ERR_ARG, "NULL argument");
    CU(cudaSetDevice(h->device));
    GroupArgs g{h->B, n_groups, h->n, counts, idx, grp_ptr};
    const int64_t work = (int64_t)h->B * n_groups;
    k_group_rates<<<(unsigned)((work + 127) / 128), 128, 0, (cudaStream_t)stream>>>(g, w, a, hz, rates);
    CU(cudaGetLastError());
    return FB_OK;
}

extern "C" int fb_clamp(fb_brain* h, const int32_t* counts, const int32_t* idx, const int32_t* grp_ptr, int32_t n_groups,
                        const int32_t* slot, const float* base, double a, double hz, float gain, float limit,
                        float* rate, float* u, const float* target, const uint8_t* active, const float* gate,
                        void* stream)
{
    if (!h || !counts || !idx || !grp_ptr || !slot || !base || !rate || !u || !target || !active || n_groups <= 0)
        return fail(FB_ERR_ARG, "NULL argument");
    CU(cudaSetDevice(h->device));
    GroupArgs g{h->B, n_groups, h->n, counts, idx, grp_ptr};
    ClampArgs c{a, hz, gain, limit, rate, u, target, active, gate, slot, base, h->bias_ext, (int32_t)h->n_ext};
    const int64_t work = (int64_t)h->B * n_groups;
    k_clamp<<<(unsigned)((work + 127) / 128), 128, 0, (cudaStream_t)stream>>>(g, c);
    CU(cudaGetLastError());
    return FB_OK;
}

extern "C" int fb_trace_rates(const fb_brain* h, const int32_t* counts, const int32_t* upre, int32_t n_upre, float* trace,
                              float a_pre, float scale_pre, const int32_t* upost, int32_t n_upost, float* rate,
                              float a_rate, float hz, void* stream)
{
    if (!h || !counts || (n_upre > 0 && (!upre || !trace)) || (n_upost > 0 && (!upost || !rate)) || n_upre < 0 ||
        n_upost < 0)
        return fail(FB_ERR_ARG, "bad arguments");
    CU(cudaSetDevice(h->device));
    const int64_t work = (int64_t)h->B * (n_upre + n_upost);
    if (work == 0) return FB_OK;
    const int blocks = (int)std::min<int64_t>((work + 255) / 256, (int64_t)h->sm_count * 8);
    k_trace_rates<<<blocks, 256, 0, (cudaStream_t)stream>>>(counts, h->n, h->B, upre, n_upre, trace, a_pre, scale_pre,
                                                            upost, n_upost, rate, a_rate, hz);
    CU(cudaGetLastError());
    return FB_OK;
}

extern "C" int fb_delta_apply(fb_brain* h, const int32_t* sel, const int32_t* pre_k, const int32_t* post_x, int32_t n_sel,
                              const float* trace, int32_t n_tr, const float* x, int32_t n_x, const float* coef,
                              const int32_t* fly_ptr, const int32_t* fly_slots, int32_t n_flies, const float* sign,
                              const float* wmax, void* stream)
{
    if (!h || n_sel < 0 || n_flies <= 0) return fail(FB_ERR_ARG, "bad arguments");
    if (n_sel == 0) return FB_OK;
    if (!sel || !pre_k || !post_x || !trace || !x || !coef || !fly_ptr || !fly_slots || !sign || !wmax)
        return fail(FB_ERR_ARG, "NULL argument");
    CU(cudaSetDevice(h->device));
    DeltaArgs a{h->B, n_flies, n_sel, n_tr, n_x, h->n_pl, sel, pre_k, post_x, trace, x, coef, fly_ptr, fly_slots, sign,
                wmax, h->pw};
    const int64_t work = (int64_t)n_sel * n_flies;
    k_delta_apply<<<(unsigned)((work + 255) / 256), 256, 0, (cudaStream_t)stream>>>(a);
    CU(cudaGetLastError());
    return FB_OK;
}

extern "C" int fb_backprop(const fb_brain* h, const int32_t* sel, const int32_t* pre_l, const int32_t* post_x, int32_t n_sel,
                           const float* x, int32_t n_x, float* delta, int32_t n_delta, void* stream)
{
    if (!h || n_sel < 0) return fail(FB_ERR_ARG, "bad arguments");
    if (n_sel == 0) return FB_OK;
    if (!sel || !pre_l || !post_x || !x || !delta) return fail(FB_ERR_ARG, "NULL argument");
    CU(cudaSetDevice(h->device));
    const int64_t work = (int64_t)h->B * n_sel;
    const int blocks = (int)std::min<int64_t>((work + 255) / 256, (int64_t)h->sm_count * 8);
    k_backprop<<<blocks, 256, 0, (cudaStream_t)stream>>>(h->B, n_sel, sel, pre_l, post_x, x, n_x, h->pw, h->n_pl,
                                                         (float)h->params.w_syn, delta, n_delta);
    CU(cudaGetLastError());
    return FB_OK;
}

extern "C" int64_t fb_eye_state_floats(int32_t batch, int32_t H, int32_t W, int32_t cell)
{
    if (batch <= 0 || cell <= 0 || H < cell || W < cell) return -1;
    const int64_t gh = H / cell, gw = W / cell;
    return (int64_t)batch * (8 * gh * gw + (gh + 1) * (gw + 1));
}

extern "C" int fb_motion_eye(fb_brain* h, const uint8_t* frames, int32_t H, int32_t W, const fb_eye_params* ep,
                             float* state, uint8_t* restart, const uint8_t* flip, int32_t n_cells, const int32_t* gx,
                             const int32_t* gy, const uint8_t* chan, const uint8_t* visible, const int32_t* slot,
                             float* rates, void* stream)
{
    if (!h || !frames || !ep || !state || !restart || n_cells < 0) return fail(FB_ERR_ARG, "NULL argument");
    if (n_cells > 0 && (!gx || !gy || !chan || !visible || !slot)) return fail(FB_ERR_ARG, "NULL argument");
    if (ep->cell <= 0 || ep->cell > 128 || H < ep->cell || W < ep->cell || ep->shift < 1 || ep->surround < 0 ||
        ep->kernels < 0 || ep->kernels > 2)
        return fail(FB_ERR_ARG, "bad eye geometry");
    CU(cudaSetDevice(h->device));
    const int32_t gh = H / ep->cell, gw = W / ep->cell;
    if (gh > 1023 || gw > 1023) return fail(FB_ERR_ARG, "eye grid wider than 1023 cells");
    const int64_t cells = (int64_t)h->B * gh * gw;
    EyeArgs a{};
    a.B = h->B; a.H = H; a.W = W; a.cell = ep->cell; a.gh = gh; a.gw = gw; a.shift = ep->shift;
    a.surround = ep->surround; a.chromatic = ep->chromatic_gain > 0.0;
    a.a_hp = ep->a_hp; a.a_d = ep->a_d; a.gain_f = (float)ep->gain; a.max_rate = (float)ep->max_rate;
    a.p_scale = ep->p_scale; a.transient_f = (float)ep->transient_gain; a.chromatic_f = (float)ep->chromatic_gain;
    a.gain = ep->gain; a.sustained = ep->sustained_gain;
    a.frames = frames; a.flip = flip; a.restart = restart;
    a.lum = state; a.lp = a.lum + cells; a.sig = a.lp + cells; a.dly = a.sig + 2 * cells; a.col = a.dly + 2 * cells;
    a.ii = a.col + 2 * cells;
    a.n_cells = n_cells; a.gx = gx; a.gy = gy; a.chan = chan; a.visible = visible; a.slot = slot;
    a.p_ext = h->p_ext; a.n_ext = (int32_t)h->n_ext; a.rates = rates;
    cudaStream_t st = (cudaStream_t)stream;
    const EyeSmem L{gh * gw, (gh + 1) * (gw + 1), a.chromatic ? 1 : 0, ep->sustained_gain != 0.0 ? 1 : 0};
    const size_t smem = L.bytes();
    const bool fits = smem <= 227 * 1024;
    if (ep->kernels == 1 && !fits) return fail(FB_ERR_ARG, "eye grid too large for the one-block-per-instance kernel");
    if (ep->kernels != 2 && fits) {
        const bool vec4 = ep->cell == 4 && W % 4 == 0 && ((uintptr_t)frames & 3) == 0;
        const void* fn = vec4 ? (const void*)k_eye_fused<true> : (const void*)k_eye_fused<false>;
        CU(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        if (vec4)
            k_eye_fused<true><<<h->B, 1024, smem, st>>>(a, L);
        else
            k_eye_fused<false><<<h->B, 1024, smem, st>>>(a, L);
        CU(cudaGetLastError());
        h->launches += 1;
        return FB_OK;
    }
    int launches = 2;
    k_eye_cells<<<(unsigned)((cells + 255) / 256), 256, 0, st>>>(a);
    if (ep->sustained_gain != 0.0) {
        const int t = ((std::max(gh, gw) + 1 + 31) / 32) * 32;
        k_eye_integral<<<h->B, t, 0, st>>>(a);
        launches++;
    }
    if (n_cells > 0) {
        const int64_t work = (int64_t)h->B * n_cells;
        k_eye_rates<<<(unsigned)((work + 255) / 256), 256, 0, st>>>(a);
        launches++;
    }
    k_eye_delay<<<(unsigned)((2 * cells + 255) / 256), 256, 0, st>>>(a);
    CU(cudaGetLastError());
    h->launches += launches;
    return FB_OK;
}

extern "C" int fb_set_schedule(fb_brain* h, int32_t engine, int32_t propagation, int32_t lanes)
{
    if (!h) return fail(FB_ERR_ARG, "NULL brain");
    if (engine < 0 || engine > FB_ENGINE_PERSISTENT) return fail(FB_ERR_ARG, "engine %d", engine);
    if (propagation != FB_PROP_PUSH && propagation != FB_PROP_PULL && propagation != -1)
        return fail(FB_ERR_ARG, "propagation %d", propagation);
    if (lanes != 0 && lanes != 8 && lanes != 16 && lanes != 32) return fail(FB_ERR_ARG, "lanes must be 8, 16 or 32");
    if (engine == FB_ENGINE_PERSISTENT && h->plan.group == 0)
        return fail(FB_ERR_UNSUPPORTED, "the persistent engine cannot hold one instance of %lld neurons on chip", (long long)h->n);
    const int new_prop = propagation >= 0 ? propagation : h->prop;
    const int new_engine = (engine != 0 || h->engine != 0) ? engine : h->engine;
    if (new_prop == FB_PROP_PULL && new_engine == FB_ENGINE_PERSISTENT)
        return fail(FB_ERR_UNSUPPORTED, "pull propagation runs on the step engine only");
    if (new_prop == FB_PROP_PULL && !h->masks) {
        CU(cudaSetDevice(h->device));
        CU(cudaDeviceSynchronize());
        int rc = enable_pull(h);
        if (rc) return rc;
    }
    if (engine != 0 || h->engine != 0) h->engine = engine;
    if (propagation >= 0) h->prop = propagation;
    if (lanes) h->lanes = lanes;
    return FB_OK;
}

extern "C" int fb_set_trace(fb_brain* h, long long* trace, int64_t capacity)
{
    if (!h) return fail(FB_ERR_ARG, "NULL brain");
    if (trace && capacity <= 0) return fail(FB_ERR_ARG, "capacity must be > 0");
    h->trace = trace;
    h->trace_cap = trace ? capacity : 0;
    return FB_OK;
}

extern "C" int fb_set_limits(fb_brain* h, int64_t barrier_cycles, int64_t item_capacity)
{
    if (!h) return fail(FB_ERR_ARG, "NULL brain");
    if (barrier_cycles < 0 || item_capacity < 0 || item_capacity > h->cap_alloc)
        return fail(FB_ERR_ARG, "barrier_cycles %lld and item_capacity %lld must be >= 0, the capacity at most %lld",
                    (long long)barrier_cycles, (long long)item_capacity, (long long)h->cap_alloc);
    h->barrier_cycles = barrier_cycles ? (long long)barrier_cycles : BARRIER_TIMEOUT_CYCLES;
    h->cap_c = item_capacity ? item_capacity : h->cap_alloc;
    return FB_OK;
}

extern "C" int fb_check(fb_brain* h, void* stream)
{
    if (!h) return fail(FB_ERR_ARG, "NULL brain");
    CU(cudaSetDevice(h->device));
    CU(cudaStreamSynchronize((cudaStream_t)stream));
    const int32_t over = h->err_h[0], tmo = h->err_h[1];
    h->err_h[0] = h->err_h[1] = 0;
    if (over) return fail(FB_ERR_OVERFLOW, "spike work list overflowed its capacity of %lld items", (long long)h->cap_c);
    if (tmo) return fail(FB_ERR_TIMEOUT, "a grid-barrier wait ran out of its budget (step %d)", tmo);
    return FB_OK;
}

namespace {

template <typename Real, typename AccT>
void launch_update(fb_brain* h, const StepArgs& A, bool raster, bool plastic, bool record, int blocks, cudaStream_t st)
{
    const DevNet N = h->net();
    const DevState S = h->state();
#define L_(R_, P_, C_) k_update<Real, AccT, R_, P_, C_><<<blocks, 256, 0, st>>>(N, S, A)
    if (raster) {
        if (plastic) { if (record) L_(true, true, true); else L_(true, true, false); }
        else { if (record) L_(true, false, true); else L_(true, false, false); }
    } else {
        if (plastic) { if (record) L_(false, true, true); else L_(false, true, false); }
        else { if (record) L_(false, false, true); else L_(false, false, false); }
    }
#undef L_
}

int dispatch_step(fb_brain* h, const StepArgs& A, bool raster, bool record, cudaStream_t st)
{
    const int64_t total = (int64_t)h->B * h->n;
    const int blocks = (int)std::min<int64_t>((total + 255) / 256, (int64_t)h->sm_count * 16);
    const bool plastic = h->n_pl > 0;
    if (h->f64) {
        if (h->acc_mode == 0) launch_update<double, int32_t>(h, A, raster, plastic, record, blocks, st);
        else launch_update<double, int64_t>(h, A, raster, plastic, record, blocks, st);
    } else {
        if (h->acc_mode == 0) launch_update<float, int32_t>(h, A, raster, plastic, record, blocks, st);
        else launch_update<float, int64_t>(h, A, raster, plastic, record, blocks, st);
    }
    CU(cudaGetLastError());
    h->launches += 1;
    return FB_OK;
}

template <typename AccT> void launch_push(fb_brain* h, int64_t t, int do_push, int blocks, cudaStream_t st)
{
    const DevNet N = h->net();
    const DevState S = h->state();
    if (h->lanes == 8) k_push<AccT, 8><<<blocks, 256, 0, st>>>(N, S, t, do_push);
    else if (h->lanes == 16) k_push<AccT, 16><<<blocks, 256, 0, st>>>(N, S, t, do_push);
    else k_push<AccT, 32><<<blocks, 256, 0, st>>>(N, S, t, do_push);
}

int dispatch_pull(fb_brain* h, int64_t t, cudaStream_t st)
{
    const int64_t work = h->n * h->mask_words;
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((work + 255) / 256, (int64_t)h->sm_count * 16));
    const DevNet N = h->net();
    const DevState S = h->state();
    if (h->acc_mode == 0) k_pull<int32_t><<<blocks, 256, 0, st>>>(N, S, t);
    else k_pull<int64_t><<<blocks, 256, 0, st>>>(N, S, t);
    CU(cudaGetLastError());
    h->launches += 1;
    return FB_OK;
}

int dispatch_push(fb_brain* h, int64_t t, cudaStream_t st)
{
    const int blocks = (int)std::min<int64_t>(std::max<int64_t>(h->sm_count, (int64_t)h->B * 16), (int64_t)h->sm_count * 8);
    const int do_push = t + 1 >= h->pushed_until;      // else pushed ahead by the persistent engine
    if (h->acc_mode == 0) launch_push<int32_t>(h, t, do_push, blocks, st);
    else launch_push<int64_t>(h, t, do_push, blocks, st);
    CU(cudaGetLastError());
    h->launches += 1;
    return FB_OK;
}

}  // namespace

extern "C" int fb_run(fb_brain* h, int32_t steps, int32_t* counts_out, const uint32_t* kicks, int32_t* step_counts,
                      uint64_t* step_digest, void* stream)
{
    if (!h || !counts_out) return fail(FB_ERR_ARG, "NULL argument");
    if (steps < 0) return fail(FB_ERR_ARG, "steps=%d", steps);
    if (kicks && h->n_ext == 0) return fail(FB_ERR_ARG, "a kick raster needs ext slots");
    CU(cudaSetDevice(h->device));
    cudaStream_t st = (cudaStream_t)stream;
    CU(cudaMemsetAsync(counts_out, 0, (size_t)h->B * h->n * sizeof(int32_t), st));
    if (step_counts) CU(cudaMemsetAsync(step_counts, 0, (size_t)steps * h->B * sizeof(int32_t), st));
    if (step_digest) CU(cudaMemsetAsync(step_digest, 0, (size_t)steps * h->B * sizeof(uint64_t), st));
    if (steps == 0) return FB_OK;
    const bool record = step_counts || step_digest;
    const int32_t words = (int32_t)((h->n_ext + 31) / 32);
    int engine = h->engine;
    if (engine == FB_ENGINE_AUTO)
        engine = (h->plan.group > 0 && !h->f64 && h->prop == FB_PROP_PUSH) ? FB_ENGINE_PERSISTENT : FB_ENGINE_STEP;
    if (engine == FB_ENGINE_PERSISTENT && h->plan.group > 0 && !h->f64) {
        h->masks_dirty = h->masks != nullptr;     // no spike masks recorded for these steps
        PersistArgs P{};
        P.t0 = h->t; P.step0 = h->step_no; P.steps = steps; P.kicks = kicks; P.words = words;
        P.counts = counts_out; P.step_counts = step_counts; P.step_digest = step_digest;
        P.bar = h->bar; P.abort_flag = h->abort_flag; P.ext_tab = h->ext_tab; P.ext_off = h->ext_off;
        P.trace = ((int64_t)steps * h->plan.ctas * TRACE_SLOTS <= h->trace_cap) ? h->trace : nullptr;
        P.pushed_until = h->pushed_until;
        P.epoch = h->epoch;
        P.barrier_cycles = h->barrier_cycles;
        CU(cudaMemsetAsync(h->abort_flag, 0, sizeof(int32_t), st));
        int rc = launch_persistent(h->plan, h->net(), h->state(), P, h->acc_mode, h->n_pl > 0 ? h->pl_mode : 0,
                                   kicks != nullptr, record, h->lanes, st);
        if (rc) return fail(FB_ERR_CUDA, "persistent launch: %s", cudaGetErrorString((cudaError_t)rc));
        h->launches += h->plan.launches_per_run;
        h->pushed_until = std::max<int64_t>(h->pushed_until, h->t + steps + 1);
    } else {
        if (h->masks && h->masks_dirty) {          // masks restart empty from this step on
            CU(cudaMemsetAsync(h->masks, 0, (size_t)h->R * h->n * h->mask_words * sizeof(unsigned long long), st));
            h->mask_from = h->t;
            h->masks_dirty = false;
        }
        for (int32_t s = 0; s < steps; s++) {
            StepArgs A{};
            A.t = h->t + s; A.step_no = h->step_no + (uint32_t)s; A.s = s; A.kicks = kicks; A.words = words;
            A.counts = counts_out; A.step_counts = step_counts; A.step_digest = step_digest;
            int rc = dispatch_step(h, A, kicks != nullptr, record, st);
            if (rc) return rc;
            // pull only for spike steps whose masks were recorded (else the work items serve)
            const bool pull = h->prop == FB_PROP_PULL && h->masks && A.t + 1 - h->n_delay >= h->mask_from &&
                              A.t + 1 >= h->pushed_until;
            rc = pull ? dispatch_pull(h, A.t, st) : dispatch_push(h, A.t, st);
            if (rc) return rc;
            h->pushed_until = std::max<int64_t>(h->pushed_until, A.t + 2);
        }
    }
    h->t += steps;
    h->step_no += (uint32_t)steps;
    return FB_OK;
}
