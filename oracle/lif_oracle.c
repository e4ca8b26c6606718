/* CPU oracle for the whole-brain LIF step. TEST INFRASTRUCTURE ONLY: the test suite, the smoke
 * check and the CPU-baseline leg of the benchmark call it as the checker; the engine never does.
 *
 * Two families of entry points (bodies in lif_oracle_impl.h, once per precision):
 *   fbo_ref_run_{f32,f64}    - flyzero/brain.py:32-58 restated statement for statement
 *                              (float summation of CSR entries in spike order);
 *   fbo_engine_run_{f32,f64} - the batched engine's semantics (exact INT32 / Q32.32 synaptic
 *                              accumulation, ext slots, plastic weights, raster or hash kicks),
 *                              which the CUDA engine must reproduce bit for bit.
 * Plus a threaded driver that runs independent instances on all cores, the reference's own
 * scaling model (one fly per process, flyzero/train.py:117-126).
 *
 * Pinned against the reference's numba kernel by tests/golden (see make_golden.py there).
 * Build: oracle/Makefile (gcc -O2 -ffp-contract=off -fno-fast-math -fPIC -shared).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define FBO_Q32_INV 2.3283064365386962890625e-10 /* 2^-32 */

#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)

typedef struct {
    int64_t n, nnz, B;
    int32_t n_delay, n_ref;
    int32_t acc_mode; /* 0: int16 counts into int32; 1: Q32.32 weights into int64 */
    int32_t contract; /* 1: fuse the two multiply-adds of the step (see lif_oracle_impl.h) */
    const int64_t* indptr;
    const int32_t* indices;
    const int16_t* cnt; /* acc_mode 0: signed synapse counts */
    const int64_t* wfx; /* acc_mode 1: q32(f32(count * w_syn)) */
    int64_t n_pl;
    const int64_t* pl_indptr; /* (n+1) plastic entries grouped by presynaptic neuron */
    const int32_t* pl_post;   /* (n_pl) postsynaptic neuron of each plastic entry */
    const int64_t* pl_q0;     /* (n_pl) q32 of the entry's connectome weight f32(count * w_syn) */
    const uint8_t* is_ppost;  /* (n) 1 where the neuron receives plastic input */
    float decay_syn_f32, decay_m_f32, kick_f32, w_syn_f32, v_rest_f32, v_th_f32, v_reset_f32;
    double decay_syn_f64, decay_m_f64, kick_f64, w_syn_f64, v_rest_f64, v_th_f64, v_reset_f64;
} fbo_net;

/* Order-independent raster fingerprint: a step's digest is the wrapping sum of this tag over
 * its spiking neurons (splitmix64 finaliser, Steele, Lea & Flood 2014). */
static inline uint64_t fbo_spike_tag(uint64_t i)
{
    uint64_t z = i + 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

/* The 32-bit integer hash used by the reference GPU engine for its Poisson draws
 * (flyzero/gpu.py:29-31; the "lowbias32" constants of Wellons' hash-prospector). */
static inline uint32_t fbo_mix32(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

/* float weight -> Q32.32, round to nearest even (x * 2^32 is exact in float). */
static inline int64_t fbo_q32(float w) { return (int64_t)llrintf(w * 4294967296.0f); }

uint64_t fbo_spike_tag_export(uint64_t i) { return fbo_spike_tag(i); }
uint32_t fbo_mix32_export(uint32_t x) { return fbo_mix32(x); }
int64_t fbo_q32_export(float w) { return fbo_q32(w); }

#define REAL float
#define SFX f32
#define FMA fmaf
#include "lif_oracle_impl.h"
#undef REAL
#undef SFX
#undef FMA

#define REAL double
#define SFX f64
#define FMA fma
#include "lif_oracle_impl.h"
#undef REAL
#undef SFX
#undef FMA

/* ------------------------------------------------------------------------------------------
 * Threaded CPU baseline: `n_inst` independent single-instance reference runs (float32,
 * brain.py:32-58) spread over `threads` POSIX threads; each instance has private state and its
 * own kick raster rows (or all share one raster). Returns the number of instances completed.
 * ------------------------------------------------------------------------------------------ */
typedef struct {
    int64_t steps, n, n_in;
    int32_t n_delay;
    const int64_t* indptr;
    const int32_t* indices;
    const float* data;
    const int64_t* input_idx;
    const uint32_t* kicks; /* (n_inst, steps, words), or (steps, words) shared when shared_kicks */
    int32_t shared_kicks;
    float kick, decay_syn, decay_m, v_rest, v_th, v_reset;
    int16_t n_ref;
    int64_t next, n_inst;
    int64_t spikes;
    pthread_mutex_t mu;
} fbo_pool_job;

static void* fbo_pool_worker(void* arg)
{
    fbo_pool_job* J = (fbo_pool_job*)arg;
    const int64_t n = J->n, words = (J->n_in + 31) / 32;
    float* v = (float*)malloc(sizeof(float) * n);
    float* g = (float*)calloc(n, sizeof(float));
    int16_t* ref = (int16_t*)calloc(n, sizeof(int16_t));
    float* pending = (float*)calloc((size_t)J->n_delay * n, sizeof(float));
    int32_t* counts = (int32_t*)calloc(n, sizeof(int32_t));
    float* bias = (float*)calloc(n, sizeof(float));
    int64_t local_spikes = 0;
    for (;;) {
        pthread_mutex_lock(&J->mu);
        int64_t k = J->next++;
        pthread_mutex_unlock(&J->mu);
        if (k >= J->n_inst) break;
        for (int64_t i = 0; i < n; i++) v[i] = J->v_rest;
        memset(g, 0, sizeof(float) * n);
        memset(ref, 0, sizeof(int16_t) * n);
        memset(pending, 0, sizeof(float) * (size_t)J->n_delay * n);
        memset(counts, 0, sizeof(int32_t) * n);
        fbo_ref_run_f32(J->steps, 0, J->n_delay, n, v, g, ref, pending, counts, J->indptr, J->indices,
                        J->data, J->input_idx, J->n_in, J->kicks + (J->shared_kicks ? 0 : k * J->steps * words), J->kick,
                        J->decay_syn, J->decay_m, J->v_rest, J->v_th, J->v_reset, J->n_ref, bias,
                        1, NULL, NULL);
        for (int64_t i = 0; i < n; i++) local_spikes += counts[i];
    }
    pthread_mutex_lock(&J->mu);
    J->spikes += local_spikes;
    pthread_mutex_unlock(&J->mu);
    free(v); free(g); free(ref); free(pending); free(counts); free(bias);
    return NULL;
}

int64_t fbo_ref_pool_f32(int32_t threads, int64_t n_inst, int64_t steps, int32_t n_delay, int64_t n,
                         const int64_t* indptr, const int32_t* indices, const float* data,
                         const int64_t* input_idx, int64_t n_in, const uint32_t* kicks, float kick,
                         float decay_syn, float decay_m, float v_rest, float v_th, float v_reset,
                         int16_t n_ref, int32_t shared_kicks, int64_t* total_spikes)
{
    fbo_pool_job J;
    memset(&J, 0, sizeof(J));
    J.steps = steps; J.n = n; J.n_in = n_in; J.n_delay = n_delay;
    J.indptr = indptr; J.indices = indices; J.data = data; J.input_idx = input_idx; J.kicks = kicks;
    J.kick = kick; J.decay_syn = decay_syn; J.decay_m = decay_m;
    J.v_rest = v_rest; J.v_th = v_th; J.v_reset = v_reset; J.n_ref = n_ref;
    J.next = 0; J.n_inst = n_inst; J.spikes = 0; J.shared_kicks = shared_kicks;
    pthread_mutex_init(&J.mu, NULL);
    if (threads < 1) threads = 1;
    pthread_t* tid = (pthread_t*)malloc(sizeof(pthread_t) * threads);
    for (int32_t k = 0; k < threads; k++) pthread_create(&tid[k], NULL, fbo_pool_worker, &J);
    for (int32_t k = 0; k < threads; k++) pthread_join(tid[k], NULL);
    free(tid);
    pthread_mutex_destroy(&J.mu);
    if (total_spikes) *total_spikes = J.spikes;
    return n_inst;
}
