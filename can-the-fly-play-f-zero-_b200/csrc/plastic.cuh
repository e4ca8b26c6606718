// The reward-modulated plastic-synapse rule on the device (traces, update, running means: three
// launches per frame):
//
//   flyzero/learning.py:116-131 (one instance, RewardPlasticity.step) and flyzero/batch.py:158-172,
//   482-495 (BatchReward.step with _Plastic.apply; flyzero/school.py:289-304 with per-slot rates):
//     dev  = c[post] - <post>                       (float32)
//     E    = ae * E + c[pre] * dev                  (E float64, c[pre]*dev float32)
//     dw_b = coef_b * E_b                           (coef_b = eta * advantage, as the rule rounds it)
//     per fly f: s_f = sum over its learning slots of f32(1/n_f) * dw_b      (the onehot GEMM)
//     every slot b of fly f: w = sign * clip(sign * (w + s_f), 0, wmax)      (float64, stored f32)
//     <post> += ap * (c[post] - <post>)             (float32 state, float64 arithmetic)
//   with sign = sign(w0), wmax = f32(cap) * max(|w0|, f32(w_syn)) in float32 (learning.py:102-104).
// Every operation is an explicit-rounding intrinsic so the result is bit-exact to NumPy's for one
// instance; for several slots of a fly only the summation order of s_f may differ (slot order here).
#pragma once
#include "common.cuh"

namespace fb {

struct RewardArgs {
    int32_t B, n_flies;
    int64_t n, n_pl;
    int32_t n_ppost;
    const int32_t* counts;       // (B, n)
    const int32_t* pre;          // (n_pl) presynaptic neuron of each plastic entry
    const int32_t* post;         // (n_pl) postsynaptic neuron
    const int32_t* pidx;         // (n_pl) compact target index
    const int32_t* ppost_neuron; // (n_ppost) neuron of each compact target
    const float* w0;             // (n_pl)
    float* pw;                   // (B, n_pl)
    double* elig;                // (B, n_pl)
    float* post_mean;            // (B, n_ppost)
    const double* coef;          // (B)
    const int32_t* fly_ptr;      // (n_flies + 1) slots grouped by fly
    const int32_t* fly_slots;    // (B)
    const float* fly_weight;     // (B) f32(1/n_active) of a learning slot, else 0
    const uint8_t* mask;         // (n_pl) entries this rule owns, or nullptr for all
    double ae, ap;
    float cap, w_syn;
    int32_t apply;
};

// the traces: one thread per (instance b, plastic entry k), b-major so that a warp's E and
// counts of one instance are contiguous
__global__ void __launch_bounds__(256) k_reward_elig(const RewardArgs a)
{
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (int64_t)a.B * a.n_pl) return;
    const int32_t b = (int32_t)(p / a.n_pl);
    const int64_t k = p - (int64_t)b * a.n_pl;
    if (a.mask && !a.mask[k]) return;
    const float c_pre = __int2float_rn(a.counts[(int64_t)b * a.n + a.pre[k]]);
    const float c_post = __int2float_rn(a.counts[(int64_t)b * a.n + a.post[k]]);
    const float dev = __fsub_rn(c_post, a.post_mean[(int64_t)b * a.n_ppost + a.pidx[k]]);
    double* e = a.elig + p;
    *e = __dadd_rn(__dmul_rn(a.ae, *e), (double)__fmul_rn(c_pre, dev));
}

// the per-fly averaged update and the clip: one thread per (fly f, plastic entry k); the fly's
// slots are summed in slot order
__global__ void __launch_bounds__(256) k_reward_apply(const RewardArgs a)
{
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (int64_t)a.n_flies * a.n_pl) return;
    const int32_t f = (int32_t)(p / a.n_pl);
    const int64_t k = p - (int64_t)f * a.n_pl;
    if (a.mask && !a.mask[k]) return;
    const float w0 = a.w0[k];
    const float sg = w0 > 0.0f ? 1.0f : (w0 < 0.0f ? -1.0f : 0.0f);
    const double wmax = (double)__fmul_rn(a.cap, fmaxf(fabsf(w0), a.w_syn));
    const double sgd = (double)sg;
    double s = 0.0;
    for (int32_t j = a.fly_ptr[f]; j < a.fly_ptr[f + 1]; j++) {
        const int32_t b = a.fly_slots[j];
        const float wgt = a.fly_weight[b];
        if (wgt != 0.0f) s = __dadd_rn(s, __dmul_rn((double)wgt, __dmul_rn(a.coef[b], a.elig[(int64_t)b * a.n_pl + k])));
    }
    for (int32_t j = a.fly_ptr[f]; j < a.fly_ptr[f + 1]; j++) {
        const int32_t b = a.fly_slots[j];
        float* w = a.pw + (int64_t)b * a.n_pl + k;
        const double x = __dmul_rn(sgd, __dadd_rn((double)*w, s));
        *w = __double2float_rn(__dmul_rn(sgd, fmin(fmax(x, 0.0), wmax)));
    }
}

__global__ void __launch_bounds__(256) k_reward_post_mean(const RewardArgs a)
{
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (int64_t)a.B * a.n_ppost) return;
    const int32_t b = (int32_t)(p / a.n_ppost), q = (int32_t)(p - (int64_t)b * a.n_ppost);
    const float c = __int2float_rn(a.counts[(int64_t)b * a.n + a.ppost_neuron[q]]);
    const float pm = a.post_mean[p];
    a.post_mean[p] = __double2float_rn(__dadd_rn((double)pm, __dmul_rn(a.ap, (double)__fsub_rn(c, pm))));
}

}  // namespace fb
