// Instructed (delta-rule) plasticity at frame ends, the drop-in for flyzero/batch.py:226-451
// (BatchInstruct, BatchInstructDeep, BatchInstructDeep2):
//
//   traces:   trace[b][k] += a_pre * (c[b][upre_k] * scale_pre - trace[b][k])        (float32)
//             rate[b][k]  += a_rate * (c[b][upost_k] * hz - rate[b][k])
//   update:   for a set of plastic synapses s (sel), per fly f:
//               d_f[s] = sum over slots b of f: coef_b * trace[b][pre_k[s]] * x[b][post_x[s]]
//             every slot b of fly f:  w = sign * clip(sign * (w + d_f[s]), 0, wmax)
//             (coef_b = eta_b / learning slots of its fly for a learning slot, else 0: the onehot
//             average of batch.py:158-172, or the deep_update kernel's coefficient, batch.py:401-404)
//   backprop: delta[b][pre_l[s]] += (pw[b][sel[s]] / w_syn) * x[b][post_x[s]]      (float atomics,
//             like the reference's scatter_add: the summation order is not fixed)
//
// With x = the DN error (target - rate) the update is the DN synapses' delta rule; with x = the
// retrograde error of layer 1 (2) it is the deep update of the layer behind it.
#pragma once
#include "common.cuh"

namespace fb {

__global__ void k_trace_rates(const int32_t* counts, int64_t n, int32_t B, const int32_t* upre, int32_t n_upre, float* trace,
                              float a_pre, float scale_pre, const int32_t* upost, int32_t n_upost, float* rate, float a_rate,
                              float hz)
{
    const int64_t total = (int64_t)B * (n_upre + n_upost);
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < total; p += (int64_t)gridDim.x * blockDim.x) {
        const int32_t b = (int32_t)(p / (n_upre + n_upost));
        const int32_t k = (int32_t)(p - (int64_t)b * (n_upre + n_upost));
        if (k < n_upre) {
            float* t = trace + (int64_t)b * n_upre + k;
            const float c = (float)counts[(int64_t)b * n + upre[k]];
            *t = __fadd_rn(*t, __fmul_rn(a_pre, __fsub_rn(__fmul_rn(c, scale_pre), *t)));
        } else {
            const int32_t q = k - n_upre;
            float* r = rate + (int64_t)b * n_upost + q;
            const float c = (float)counts[(int64_t)b * n + upost[q]];
            *r = __fadd_rn(*r, __fmul_rn(a_rate, __fsub_rn(__fmul_rn(c, hz), *r)));
        }
    }
}

struct DeltaArgs {
    int32_t B, n_flies, n_sel, n_tr, n_x;
    int64_t n_pl;
    const int32_t* sel;        // (n_sel) plastic entry of each synapse of the set
    const int32_t* pre_k;      // (n_sel) its presynaptic trace index
    const int32_t* post_x;     // (n_sel) its column of x
    const float* trace;        // (B, n_tr)
    const float* x;            // (B, n_x)
    const float* coef;         // (B)
    const int32_t* fly_ptr;    // (n_flies + 1) slots of each fly: fly_slots[fly_ptr[f] .. fly_ptr[f+1])
    const int32_t* fly_slots;
    const float* sign;         // (n_pl)
    const float* wmax;         // (n_pl)
    float* pw;                 // (B, n_pl)
};

// one thread per (synapse of the set, fly)
__global__ void k_delta_apply(const DeltaArgs a)
{
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (int64_t)a.n_sel * a.n_flies) return;
    const int32_t s = (int32_t)(p / a.n_flies), f = (int32_t)(p - (int64_t)s * a.n_flies);
    const int32_t j = a.sel[s], pk = a.pre_k[s], px = a.post_x[s];
    float d = 0.0f;
    for (int32_t q = a.fly_ptr[f]; q < a.fly_ptr[f + 1]; q++) {
        const int32_t b = a.fly_slots[q];
        const float c = a.coef[b];
        if (c != 0.0f)
            d = __fadd_rn(d, __fmul_rn(__fmul_rn(c, a.trace[(int64_t)b * a.n_tr + pk]), a.x[(int64_t)b * a.n_x + px]));
    }
    if (d == 0.0f) return;
    const float sg = a.sign[j], mx = a.wmax[j];
    for (int32_t q = a.fly_ptr[f]; q < a.fly_ptr[f + 1]; q++) {
        float* w = a.pw + (int64_t)a.fly_slots[q] * a.n_pl + j;
        const float v = __fmul_rn(sg, __fadd_rn(*w, d));
        *w = __fmul_rn(sg, fminf(fmaxf(v, 0.0f), mx));
    }
}

__global__ void k_backprop(int32_t B, int32_t n_sel, const int32_t* sel, const int32_t* pre_l, const int32_t* post_x,
                           const float* x, int32_t n_x, const float* pw, int64_t n_pl, float w_syn, float* delta,
                           int32_t n_delta)
{
    const int64_t total = (int64_t)B * n_sel;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < total; p += (int64_t)gridDim.x * blockDim.x) {
        const int32_t b = (int32_t)(p / n_sel), s = (int32_t)(p - (int64_t)b * n_sel);
        const float v = __fmul_rn(__fdiv_rn(pw[(int64_t)b * n_pl + sel[s]], w_syn), x[(int64_t)b * n_x + post_x[s]]);
        atomicAdd(delta + (int64_t)b * n_delta + pre_l[s], v);
    }
}

}  // namespace fb
