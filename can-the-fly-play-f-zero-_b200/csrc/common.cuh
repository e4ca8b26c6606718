// Device-side building blocks of the LIF engine: exact-rounding arithmetic, the Poisson hash,
// the raster fingerprint and the per-instance-neuron step. Every floating-point operation of the
// step is spelled out with an explicit-rounding intrinsic so that nvcc cannot contract or
// reorder it: the engine must reproduce the CPU oracle bit for bit.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace fb {

constexpr int CHUNK = 256;          // CSR entries per spike work item (flyzero/gpu.py:72-81 uses 256 too)
constexpr int CHUNK_BITS = 12;      // item.y = (instance << 12) | chunk
constexpr int EDGE_ALIGN = 8;       // device CSR rows are padded to multiples of 8 entries (16 B of int16)
constexpr double Q32_INV = 2.3283064365386962890625e-10;   // 2^-32

// ---- explicit-rounding arithmetic, overloaded on the state type ----------------------------
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }

template <typename Real> __device__ __forceinline__ Real from_q32(int64_t x);
template <> __device__ __forceinline__ float from_q32<float>(int64_t x)
{
    return __double2float_rn(__dmul_rn(__ll2double_rn(x), Q32_INV));
}
template <> __device__ __forceinline__ double from_q32<double>(int64_t x)
{
    return __dmul_rn(__ll2double_rn(x), Q32_INV);
}

// synaptic input of one step from the accumulator: INT32 counts scaled once, or Q32.32
template <typename Real> __device__ __forceinline__ Real acc_to_real(int32_t x, Real w_syn)
{
    return mul_rn((Real)x, w_syn);   // int32 -> float is exact below 2^24, -> double always
}
template <typename Real> __device__ __forceinline__ Real acc_to_real(int64_t x, Real)
{
    return from_q32<Real>(x);
}

// float weight -> Q32.32 (x * 2^32 is exact in float; conversion rounds half to even)
__device__ __forceinline__ int64_t to_q32(float w) { return __float2ll_rn(__fmul_rn(w, 4294967296.0f)); }

// The reference GPU engine's 32-bit hash (flyzero/gpu.py:29-31), constants of the "lowbias32"
// function from Wellons' hash-prospector. Kept so that equal seeds give the reference's noise.
__device__ __forceinline__ uint32_t mix32(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

// One Poisson draw per (instance, neuron, step), as flyzero/gpu.py:63-69 draws it.
__device__ __forceinline__ bool hash_kick(uint32_t tid, uint32_t step_no, uint32_t seed, uint32_t b, float p)
{
    uint32_t h = mix32(tid ^ mix32(step_no * 0x9e3779b9u ^ mix32(seed + b)));
    return __fmul_rn(__uint2float_rn(h >> 8), 1.0f / 16777216.0f) < p;
}

// Raster fingerprint tag of neuron i (splitmix64 finaliser; Steele, Lea & Flood 2014).
__device__ __forceinline__ uint64_t spike_tag(uint64_t i)
{
    uint64_t z = i + 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

template <typename Real> struct Lif {
    Real ds, dm, kick, w_syn, v_rest, v_th, v_reset;
};

// The step of one instance-neuron (flyzero/brain.py:39-56 order; flyzero/gpu.py:48-70):
//   g = g*decay_syn + buf; refractory decrement or v += ((g + bias) - (v - v_rest)) * decay_m;
//   Poisson kick; spike test v >= v_th && ref <= 0; reset.
// `contract` fuses the two multiply-adds exactly where the shipped reference kernel does.
template <typename Real>
__device__ __forceinline__ bool lif_step(Real& v, Real& g, int& r, Real buf, bool has_bias, float bias,
                                         bool kicked, const Lif<Real>& L, int n_ref, bool contract)
{
    g = contract ? fma_rn(g, L.ds, buf) : add_rn(mul_rn(g, L.ds), buf);
    if (r > 0) {
        r -= 1;
    } else {
        Real a = has_bias ? add_rn(g, (Real)bias) : g;
        Real e = sub_rn(a, sub_rn(v, L.v_rest));
        v = contract ? fma_rn(e, L.dm, v) : add_rn(v, mul_rn(e, L.dm));
    }
    if (kicked) v = add_rn(v, L.kick);
    if (v >= L.v_th && r <= 0) {
        v = L.v_reset;
        r = n_ref;
        return true;
    }
    return false;
}

}  // namespace fb
