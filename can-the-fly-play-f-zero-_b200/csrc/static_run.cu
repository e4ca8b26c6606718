// fb_run_static: one LIF instance advanced without any device allocation by the library.
//
// Some callers cannot allocate device memory when they want to simulate: a host program whose
// GPU memory is entirely managed by another allocator (a framework's caching pool that must see
// every byte), a control loop that cannot afford the implicit device synchronisation of
// cudaMalloc/cudaFree in the middle of a run, or an embedded/certified deployment that forbids
// run-time allocation after start-up. For them this entry point takes every input and output as
// caller-owned device memory and keeps its only scratch - the ring of synaptic input in flight -
// in a fixed-size array compiled into the library (FB_STATIC_RING_ENTRIES int64 = 8 MiB, held by
// every GPU that loads the library until the process exits).
//
// The step is the same as the step engine's in Q32.32 mode (FB_FLAG_ACC_FIXED): weights enter as
// q32(w) and integer sums are exact, so the result equals fb_run's bit for bit. The rows of a
// step's spikes go straight into ring slot (t + n_delay) mod (n_delay + 1), one warp per spiking
// lane, inside the same launch that advanced the neurons (that slot is not read in step t).
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/flybrain.h"
#include "common.cuh"

namespace fb {

void set_last_error(const char* msg);   // flybrain.cu: the message fb_last_error() returns

// The scratch: file scope, 256-byte aligned, one per device that loads the library.
static __device__ __align__(256) int64_t g_static_ring[FB_STATIC_RING_ENTRIES];

namespace {

std::mutex g_static_mu;
void* g_static_addr[128] = {nullptr};   // device address of g_static_ring, per device ordinal

struct StaticArgs {
    int64_t n;
    int32_t n_delay, R, n_ref;
    double dt, tau_m, tau_syn, f_poisson, w_syn;
    float v_rest, v_th, v_reset;
    const int64_t* indptr;
    const int32_t* indices;
    const float* weights;
    float* v;
    float* g;
    int8_t* ref;
    const int32_t* ext_idx;
    const float* p_ext;
    const float* bias_ext;
    uint32_t seed;
    int32_t* counts;
};

__global__ void __launch_bounds__(256) k_static_step(const StaticArgs a, int64_t* ring, int64_t t, uint32_t step_no)
{
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    // constants exactly as the engine derives them: FP64 on the device, then rounded
    Lif<float> L;
    L.ds = __double2float_rn(exp(-a.dt / a.tau_syn));
    L.dm = __double2float_rn(a.dt / a.tau_m);
    L.kick = __double2float_rn(a.f_poisson * a.w_syn);
    L.w_syn = __double2float_rn(a.w_syn);
    L.v_rest = a.v_rest;
    L.v_th = a.v_th;
    L.v_reset = a.v_reset;
    // non-negative slots even for a negative tick (the host rejects t0 < 0 as well)
    const int64_t si = ((t % a.R) + a.R) % a.R, so = (((t + a.n_delay) % a.R) + a.R) % a.R;
    int64_t* in_slot = ring + si * a.n;
    int64_t* out_slot = ring + so * a.n;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < a.n; base += stride) {
        const int64_t i = base + threadIdx.x;
        bool spk = false;
        if (i < a.n) {
            const int64_t x = in_slot[i];
            if (x != 0) in_slot[i] = 0;
            const float buf = from_q32<float>(x);
            float v = a.v[i], g = a.g[i];
            int r = a.ref[i];
            const int32_t j = a.ext_idx ? a.ext_idx[i] : -1;
            float bias = 0.0f;
            bool kicked = false;
            if (j >= 0) {
                bias = a.bias_ext[j];
                const float p = a.p_ext[j];
                kicked = p > 0.0f && hash_kick((uint32_t)i, step_no, a.seed, 0u, p);
            }
            spk = lif_step<float>(v, g, r, buf, j >= 0, bias, kicked, L, a.n_ref, true);
            a.v[i] = v;
            a.g[i] = g;
            a.ref[i] = (int8_t)r;
            if (spk) a.counts[i] += 1;
        }
        // each spiking lane's row, scattered by the whole warp
        unsigned m = __ballot_sync(FULL, spk);
        while (m) {
            const int leader = __ffs(m) - 1;
            m &= m - 1;
            const int64_t row = __shfl_sync(FULL, i, leader);
            const int64_t k1 = a.indptr[row + 1];
            for (int64_t k = a.indptr[row] + lane; k < k1; k += 32) {
                const int64_t w = to_q32(a.weights[k]);
                if (w != 0) atomicAdd(reinterpret_cast<unsigned long long*>(out_slot + a.indices[k]), (unsigned long long)w);
            }
        }
    }
}

int static_fail(int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    set_last_error(buf);   // read back through fb_last_error()
    return code;
}

// Device address of the scratch for the current device, looked up once per device. A device reset
// (cudaDeviceReset, or any teardown of the primary context) reloads the module, possibly at another
// address, so the cached address is only valid for the context it was looked up in.
int static_scratch(int64_t** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return static_fail(FB_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= 128) return static_fail(FB_ERR_UNSUPPORTED, "device ordinal %d", dev);
    std::lock_guard<std::mutex> lock(g_static_mu);
    if (!g_static_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_static_ring);
        if (e != cudaSuccess || !p)
            return static_fail(FB_ERR_CUDA, "cudaGetSymbolAddress(static ring): %s", cudaGetErrorString(e));
        g_static_addr[dev] = p;
    }
    *out = reinterpret_cast<int64_t*>(g_static_addr[dev]);
    return FB_OK;
}

}  // namespace

}  // namespace fb

extern "C" int fb_run_static(const fb_params* p, int64_t n, const int64_t* indptr, const int32_t* indices,
                             const float* weights, float* v, float* g, int8_t* ref, const int32_t* ext_idx,
                             const float* p_ext, const float* bias_ext, uint32_t seed, uint32_t step_no, int64_t t0,
                             int32_t steps, int32_t clear, int32_t* counts, void* stream)
{
    using namespace fb;
    if (!p || n <= 0 || !indptr || !indices || !weights || !v || !g || !ref || !counts || steps < 0)
        return static_fail(FB_ERR_ARG, "fb_run_static: NULL pointer or bad size");
    if (ext_idx && (!p_ext || !bias_ext))
        return static_fail(FB_ERR_ARG, "fb_run_static: ext_idx needs p_ext and bias_ext");
    if (!(p->dt > 0) || !(p->tau_m > 0) || !(p->tau_syn > 0) || !std::isfinite(p->dt))
        return static_fail(FB_ERR_ARG, "fb_run_static: dt, tau_m, tau_syn must be finite and > 0");
    // ticks index the ring as t mod (n_delay + 1): they must stay non-negative for the whole call
    if (t0 < 0 || t0 > INT64_MAX - (int64_t)steps)
        return static_fail(FB_ERR_ARG, "fb_run_static: t0=%lld must be >= 0 and t0 + steps must not overflow",
                           (long long)t0);
    // delay/dt and t_ref/dt are rounded to step counts; reject values whose rounding is not a small integer
    const double dq = p->delay / p->dt, rq = p->t_ref / p->dt;
    if (!std::isfinite(dq) || !std::isfinite(rq) || std::fabs(dq) > 1e6 || rq > 1e6 || rq < -0.5)
        return static_fail(FB_ERR_ARG, "fb_run_static: delay/dt must be finite with |delay/dt| <= 1e6, t_ref/dt finite in [0, 1e6]");
    const int64_t nd = std::max<int64_t>(1, (int64_t)std::nearbyint(dq));
    const int64_t nr = (int64_t)std::nearbyint(rq);
    if (nr < 0 || nr > 127) return static_fail(FB_ERR_ARG, "fb_run_static: n_ref=%lld must fit int8", (long long)nr);
    // division, not n * (nd + 1): the product could overflow for huge n
    if (n > (int64_t)INT32_MAX - 1 || nd + 1 > (int64_t)FB_STATIC_RING_ENTRIES / n)
        return static_fail(FB_ERR_ARG,
                           "fb_run_static: n * (n_delay + 1) = %lld * %lld exceeds the static ring of %lld entries "
                           "(use fb_create/fb_run for larger networks)",
                           (long long)n, (long long)(nd + 1), (long long)FB_STATIC_RING_ENTRIES);
    int64_t* ring = nullptr;
    int rc = static_scratch(&ring);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e;
    if (clear && (e = cudaMemsetAsync(ring, 0, (size_t)n * (nd + 1) * sizeof(int64_t), st)) != cudaSuccess)
        return static_fail(FB_ERR_CUDA, "fb_run_static: clearing the ring: %s", cudaGetErrorString(e));
    if ((e = cudaMemsetAsync(counts, 0, (size_t)n * sizeof(int32_t), st)) != cudaSuccess)
        return static_fail(FB_ERR_CUDA, "fb_run_static: clearing counts: %s", cudaGetErrorString(e));
    StaticArgs a{};
    a.n = n; a.n_delay = (int32_t)nd; a.R = (int32_t)(nd + 1); a.n_ref = (int32_t)nr;
    a.dt = p->dt; a.tau_m = p->tau_m; a.tau_syn = p->tau_syn; a.f_poisson = p->f_poisson; a.w_syn = p->w_syn;
    a.v_rest = (float)p->v_rest; a.v_th = (float)p->v_th; a.v_reset = (float)p->v_reset;
    a.indptr = indptr; a.indices = indices; a.weights = weights; a.v = v; a.g = g; a.ref = ref;
    a.ext_idx = ext_idx; a.p_ext = p_ext; a.bias_ext = bias_ext; a.seed = seed; a.counts = counts;
    int sms = 148, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int blocks = (int)std::min<int64_t>((n + 255) / 256, (int64_t)sms * 8);
    for (int32_t s = 0; s < steps; s++) {
        k_static_step<<<blocks, 256, 0, st>>>(a, ring, t0 + s, step_no + (uint32_t)s);
        if ((e = cudaGetLastError()) != cudaSuccess)
            return static_fail(FB_ERR_CUDA, "fb_run_static: launch: %s", cudaGetErrorString(e));
    }
    return FB_OK;
}
