// Host launchers for the reference's own CUDA kernels `update` and `propagate` (the `_SRC` string of
// flyzero/gpu.py:26-119). Test infrastructure only: oracle/make_ref_gpu.py extracts that string from
// the reference checkout into oracle/_ref/ at build time (it is never committed) and compiles it with
// this file, so that the reference's GPU method can be timed beside the engine on the same device.
// The launch shapes are the reference's (gpu.py:239-252): `update` over B*n threads in blocks of
// 256, `propagate` on 240 blocks of 256.
#include <cuda_runtime.h>

#include REF_SRC

extern "C" int refgpu_update(int blocks, void* stream, int B, int n, int slot, unsigned int step, unsigned int seed,
                             float* v, float* g, signed char* ref, float* pending, int* counts, const int* ext_idx,
                             int n_ext, const float* p_ext, const float* bias_ext, float kick, float decay_syn,
                             float decay_m, float v_rest, float v_th, float v_reset, int n_ref, const long long* indptr,
                             const long long* pl_indptr, int* spikes, int* n_spikes)
{
    update<<<blocks, 256, 0, (cudaStream_t)stream>>>(B, n, slot, step, seed, v, g, ref, pending, counts, ext_idx, n_ext,
                                                    p_ext, bias_ext, kick, decay_syn, decay_m, v_rest, v_th, v_reset,
                                                    n_ref, indptr, pl_indptr, spikes, n_spikes);
    return (int)cudaGetLastError();
}

extern "C" int refgpu_propagate(int blocks, void* stream, int B, int n, int slot, const int* spikes, int* n_spikes,
                                int next, const long long* indptr, const int* indices, const float* data,
                                const long long* pl_indptr, const int* pl_post, const float* pl_w, int n_pl,
                                float* pending)
{
    propagate<<<blocks, 256, 0, (cudaStream_t)stream>>>(B, n, slot, spikes, n_spikes, next, indptr, indices, data,
                                                       pl_indptr, pl_post, pl_w, n_pl, pending);
    return (int)cudaGetLastError();
}
