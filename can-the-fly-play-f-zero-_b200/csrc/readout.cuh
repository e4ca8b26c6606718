// Frame-end readout of neuron groups, fused on the device: the smoothed group rates the motor
// readout (flyzero/batch.py:77-138, BatchMotor.update) and the closed-loop clamp
// (flyzero/implant.py:69-104, Clamp.step) compute from a frame's spike counts, and the clamp's
// controller writing the groups' bias. One thread per (instance, group); groups are short lists
// of neurons (a few per cell type), so the gather is a loop.
//
//   readout: inst = f32(sum_k counts[b][idx_k]) * w_g * hz       (w_g = 1 / group size, f32)
//            rate += a * (inst - rate)                             (f32, as NumPy computes it)
//   clamp:   inst = (sum_k counts[b][idx_k] / size_g) * hz         (f64, cupy's mean)
//            rate = f32(rate + a * (inst - rate))
//            u    = clip(u + gain * (target - rate) * on, -limit, limit) * active
//            bias_ext[b][slot_k] = base_k + u * on                  for every k of the group
#pragma once
#include "common.cuh"

namespace fb {

struct GroupArgs {
    int32_t B, n_groups;
    int64_t n;
    const int32_t* counts;      // (B, n)
    const int32_t* idx;         // neurons of all groups, group after group
    const int32_t* grp_ptr;     // (n_groups + 1) offsets into idx
};

__device__ __forceinline__ int64_t group_sum(const GroupArgs& g, int32_t b, int32_t k)
{
    int64_t s = 0;
    for (int32_t q = g.grp_ptr[k]; q < g.grp_ptr[k + 1]; q++) s += g.counts[(int64_t)b * g.n + g.idx[q]];
    return s;
}

__global__ void k_group_rates(const GroupArgs g, const float* w, float a, float hz, float* rates)
{
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (int64_t)g.B * g.n_groups) return;
    const int32_t b = (int32_t)(p / g.n_groups), k = (int32_t)(p - (int64_t)b * g.n_groups);
    const float inst = __fmul_rn(__fmul_rn((float)group_sum(g, b, k), w[k]), hz);
    const float r = rates[p];
    rates[p] = __fadd_rn(r, __fmul_rn(a, __fsub_rn(inst, r)));
}

struct ClampArgs {
    double a, hz;
    float gain, limit;
    float* rate;                // (B, n_groups)
    float* u;                   // (B, n_groups)
    const float* target;        // (B, n_groups)
    const uint8_t* active;      // (B)
    const float* gate;          // (B, n_groups) or nullptr (all open)
    const int32_t* slot;        // ext slot of every idx entry
    const float* base;          // (B, len(idx)) bias of every idx entry without the clamp
    float* bias_ext;            // (B, n_ext)
    int32_t n_ext;
};

__global__ void k_clamp(const GroupArgs g, const ClampArgs c)
{
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (int64_t)g.B * g.n_groups) return;
    const int32_t b = (int32_t)(p / g.n_groups), k = (int32_t)(p - (int64_t)b * g.n_groups);
    const int32_t size = g.grp_ptr[k + 1] - g.grp_ptr[k];
    const double inst = __dmul_rn(__ddiv_rn((double)group_sum(g, b, k), (double)max(size, 1)), c.hz);
    const float r = __double2float_rn(__dadd_rn((double)c.rate[p], __dmul_rn(c.a, __dsub_rn(inst, (double)c.rate[p]))));
    c.rate[p] = r;
    const float act = c.active[b] ? 1.0f : 0.0f;
    const float on = act * (c.gate ? c.gate[p] : 1.0f);
    float u = __fadd_rn(c.u[p], __fmul_rn(__fmul_rn(c.gain, __fsub_rn(c.target[p], r)), on));
    u = __fmul_rn(fminf(fmaxf(u, -c.limit), c.limit), act);
    c.u[p] = u;
    const float applied = __fmul_rn(u, on);
    const int64_t L = g.grp_ptr[g.n_groups];
    for (int32_t q = g.grp_ptr[k]; q < g.grp_ptr[k + 1]; q++)
        c.bias_ext[(int64_t)b * c.n_ext + c.slot[q]] = __fadd_rn(c.base[(int64_t)b * L + q], applied);
}

}  // namespace fb
