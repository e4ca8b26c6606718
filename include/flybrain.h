/* flybrain.h - C ABI of the B200 LIF engine (libflybrain.so).
 *
 * One engine ("brain") holds B instances ("flies") of a leaky integrate-and-fire network that
 * share one connectome. It replaces the reference's CPU engine `flyzero.brain.Brain`
 * (flyzero/brain.py:79-172) and its CuPy engine `flyzero.gpu.BatchBrain`
 * (flyzero/gpu.py:131-254); the reference binds its engines from Python, so the binding a
 * maintainer adds is a ctypes stub over these entry points.
 *
 * Conventions
 *   - Every function returns FB_OK (0) or an FB_ERR_* code; fb_last_error() gives the message
 *     of the calling thread's last failure. No C++ exception crosses this boundary.
 *   - Host pointers are marked [host], device pointers [device]. Device buffers handed out by
 *     fb_get_views() are owned by the engine and valid until the next fb_set_ext() (ext
 *     buffers only) or fb_destroy().
 *   - `stream` is a cudaStream_t (NULL = legacy default stream). All work is enqueued on it;
 *     no function synchronises the host except where stated.
 */
#ifndef FLYBRAIN_H
#define FLYBRAIN_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FB_OK 0
#define FB_ERR_ARG 1         /* invalid argument (message says which) */
#define FB_ERR_CUDA 2        /* a CUDA runtime call failed */
#define FB_ERR_OVERFLOW 3    /* the spike work list overflowed its capacity (device flag) */
#define FB_ERR_TIMEOUT 4     /* a grid-barrier wait ran out of its iteration budget (device flag) */
#define FB_ERR_UNSUPPORTED 5 /* valid request that this build does not support */

/* create() flags */
#define FB_FLAG_F64 1u           /* FP64 state: the oracle-mode step (precision reports) */
#define FB_FLAG_ACC_FIXED 2u     /* force Q32.32 fixed-point accumulation even for integer counts */

/* schedule: engine kinds */
#define FB_ENGINE_AUTO 0
#define FB_ENGINE_STEP 1         /* two launches per simulated step (update, propagate) */
#define FB_ENGINE_PERSISTENT 2   /* one persistent launch per run; state kept on chip */
/* schedule: propagation kinds */
#define FB_PROP_PUSH 0           /* scatter each spiking row into the accumulator (atomics) */
#define FB_PROP_PULL 1           /* gather per postsynaptic neuron from the spike history */

typedef struct fb_brain fb_brain;

/* LIFParams (flyzero/brain.py:65-76); derived constants follow brain.py:92-96. */
typedef struct {
    double v_rest, v_reset, v_th, tau_m, tau_syn, t_ref, delay, w_syn, f_poisson, dt;
} fb_params;

typedef struct {
    int64_t n;            /* neurons */
    int64_t nnz;          /* CSR entries */
    int32_t batch;        /* instances */
    int32_t n_delay;      /* max(1, round(delay / dt)) */
    int32_t n_ref;        /* round(t_ref / dt) */
    int32_t acc_mode;     /* 0: INT32 synapse counts, 1: INT64 Q32.32 weights */
    int32_t f64;          /* 1 for FP64 state */
    int32_t engine;       /* current schedule (FB_ENGINE_*) */
    int32_t propagation;  /* FB_PROP_* */
    int32_t lanes;        /* lanes per spike work item (8, 16 or 32) */
    int32_t group;        /* instances per persistent group (0: persistent engine unavailable) */
    int32_t ctas;         /* CTAs of the persistent launch */
    int64_t n_plastic;    /* plastic CSR entries */
    int64_t n_ext;        /* ext slots (neurons that take Poisson rates and/or bias) */
    int64_t t;            /* simulated steps since the last full reset (BatchBrain.t) */
    uint32_t step_no;     /* global step counter feeding the Poisson hash (BatchBrain.step_no) */
    int64_t launches;     /* kernels launched by this engine so far */
    int64_t item_capacity;/* spike work items per (step, instance group, list segment) list */
    int64_t bytes_device; /* device memory held by the engine */
    double decay_syn;     /* exp(-dt / tau_syn), computed in FP64 on the device */
    double decay_m;       /* dt / tau_m */
    double kick;          /* f_poisson * w_syn, mV */
    int32_t epoch;        /* persistent engine: steps between grid barriers (accumulator slots = 2x) */
} fb_info;

/* Device views of the mutable state a caller may read and write between runs. */
typedef struct {
    void* v;          /* (batch, n) float32, or float64 with FB_FLAG_F64: membrane potential, mV */
    void* g;          /* (batch, n) same type: synaptic conductance, mV */
    int8_t* ref;      /* (batch, n) refractory steps left */
    float* pw;        /* (batch, n_plastic) plastic weights in mV (already x w_syn), gpu.py:163 */
    float* w0;        /* (n_plastic) initial plastic weights */
    int32_t* ext_idx; /* (n) ext slot of each neuron or -1 (read-only) */
    float* p_ext;     /* (batch, n_ext) Poisson probability per step (rate * dt / 1000), gpu.py:226 */
    float* bias_ext;  /* (batch, n_ext) steady bias, mV (gpu.py:215-220) */
    int64_t* stop_tick; /* (batch) instance b advances only while t < stop_tick[b] */
} fb_views;

/* Create an engine. The CSR (pre x post, signed synapse counts as float32, like
 * flyzero/connectome.py:140-146) is copied to the device, sorted by column within each row.
 * plastic_pos: CSR positions (Brain.data layout) whose weight is per instance (gpu.py:150-163).
 * Replaces: Brain.__init__ (flyzero/brain.py:80-102), BatchBrain.__init__ (flyzero/gpu.py:139-184). */
int fb_create(const fb_params* params, const int64_t* indptr /*[host] n+1*/,
              const int32_t* indices /*[host] nnz*/, const float* data /*[host] nnz*/, int64_t n,
              int64_t nnz, int32_t batch, uint32_t seed, const int64_t* plastic_pos /*[host]*/,
              int64_t n_plastic, uint32_t flags, int32_t device, fb_brain** out);

int fb_destroy(fb_brain* brain);

/* Message of the calling thread's last failure (always NUL-terminated). */
int fb_last_error(char* buf, int64_t len);

int fb_get_info(const fb_brain* brain, fb_info* out);

int fb_get_views(fb_brain* brain, fb_views* out);

/* Give the neurons idx[0..count) an ext slot if they have none (BatchBrain.slots,
 * flyzero/gpu.py:201-213). Existing p_ext / bias_ext values are kept; new slots start at 0.
 * Reallocates p_ext / bias_ext: call fb_get_views() again afterwards. Synchronises the device. */
int fb_set_ext(fb_brain* brain, const int64_t* idx /*[host]*/, int64_t count);

/* Make the CSR positions pos[0..count) plastic as well (per-instance weights in pw), keeping all
 * state and the synaptic input in flight. A new plastic entry starts at its connectome weight in
 * every instance; plastic entries always enter as the delta of pw over that weight, pushed at spike
 * time, so a weight written between runs affects only later spikes (as writes to Brain.data do
 * in the reference, flyzero/learning.py:130). Reallocates pw / w0: call fb_get_views() again.
 * Synchronises the device. */
int fb_set_plastic(fb_brain* brain, const int64_t* pos /*[host]*/, int64_t count);

/* Back to rest: v = v_rest, g = 0, ref = 0 and no synaptic input in flight
 * (BatchBrain.reset, flyzero/gpu.py:186-199; Brain.reset, flyzero/brain.py:104-110).
 * flies == NULL or n_flies < 0: every instance, and t = 0. Plastic weights are kept. The list
 * of flies is copied before return (through pinned staging; the host is not synchronised with the
 * stream). */
int fb_reset(fb_brain* brain, const int32_t* flies /*[host]*/, int32_t n_flies, void* stream);

/* Advance every instance `steps` steps (BatchBrain.run, flyzero/gpu.py:228-254; Brain.run,
 * flyzero/brain.py:133-172).
 *   counts_out   [device] (batch, n) int32, overwritten with this run's spike counts.
 *   kicks        [device] NULL: Poisson kicks from the counter hash of p_ext (gpu.py:63-69);
 *                else a raster (steps, batch, ceil(n_ext/32)) uint32, bit j%32 of word j/32 =
 *                kick ext slot j at that step (parity mode: identical precomputed input spikes).
 *   step_counts  [device] NULL or (steps, batch) int32: spikes per step (overwritten).
 *   step_digest  [device] NULL or (steps, batch) uint64: order-independent raster fingerprint per
 *                step, the wrapping sum over spiking neurons i of splitmix64(i) (overwritten). */
int fb_run(fb_brain* brain, int32_t steps, int32_t* counts_out, const uint32_t* kicks,
           int32_t* step_counts, uint64_t* step_digest, void* stream);

/* The reward-modulated plastic update of every instance on the device (traces per instance and
 * entry, the update per fly and entry, the running means: three launches, two when apply is 0).
 * Restates RewardPlasticity.step (flyzero/learning.py:116-131) for one instance and
 * BatchReward.step + _Plastic.apply (flyzero/batch.py:158-172, 482-495) for many:
 *   E = ae*E + c[pre]*(c[post] - <post>);  per fly f: s_f = sum_{learning b of f} fly_weight[b]*coef[b]*E_b;
 *   every slot b of fly f: pw = sign*clip(sign*(pw + s_f), 0, cap*max(|w0|, w_syn));
 *   <post> += ap*(c[post] - <post>).
 *   counts     [device] (batch, n) int32 spike counts of the window just run
 *   elig       [device] (batch, n_plastic) float64 eligibility traces, updated in place
 *   post_mean  [device] (batch, n_targets) float32 running mean count of each plastic target
 *              (targets = distinct postsynaptic neurons of the plastic entries, ascending)
 *   coef       [device] (batch) float64: eta * advantage of each slot, rounded as the rule does
 *   fly_ptr    [device] (n_flies+1), fly_slots [device] (batch): slots grouped by fly, each slot in
 *              one fly at most (the flies' updates run in parallel)
 *   fly_weight [device] (batch) float32: 1/(learning slots of the fly) for a learning slot, else 0
 *   mask       [device] NULL or (n_plastic) uint8: the plastic entries this rule owns (others untouched)
 *   apply      0: traces and means only (no slot learns this frame, batch.py:493) */
int fb_reward_step(fb_brain* brain, const int32_t* counts, double* elig, float* post_mean, const double* coef,
                   const int32_t* fly_ptr, const int32_t* fly_slots, const float* fly_weight, int32_t n_flies,
                   const uint8_t* mask, double ae, double ap, float cap, int32_t apply, void* stream);

/* Frame-end readout of neuron groups (BatchMotor.update, flyzero/batch.py:105-109): for every
 * instance b and group g (neurons idx[grp_ptr[g] .. grp_ptr[g+1]) [device]),
 *   inst = f32(sum of counts[b][idx]) * w[g] * hz;  rates[b][g] += a * (inst - rates[b][g])
 * counts [device] (batch, n); w [device] (n_groups) = 1 / group size; rates [device] (batch,
 * n_groups) float32, updated in place. */
int fb_group_rates(const fb_brain* brain, const int32_t* counts, const int32_t* idx, const int32_t* grp_ptr,
                   int32_t n_groups, const float* w, float a, float hz, float* rates, void* stream);

/* Closed-loop clamp of neuron groups (Clamp.step, flyzero/implant.py:84-104), all on the device:
 *   rate = rate + a * (mean count * hz - rate);  on = active[b] * gate[b][g] (gate NULL: 1)
 *   u = clip(u + gain * (target - rate) * on, -limit, limit) * active[b]
 *   bias_ext[b][slot[k]] = base[b][k] + u * on     for every entry k of the group
 * slot [device] ext slot of every idx entry; base [device] (batch, len(idx)); rate, u, target,
 * gate [device] (batch, n_groups) float32; active [device] (batch) uint8. */
int fb_clamp(fb_brain* brain, const int32_t* counts, const int32_t* idx, const int32_t* grp_ptr, int32_t n_groups,
             const int32_t* slot, const float* base, double a, double hz, float gain, float limit, float* rate,
             float* u, const float* target, const uint8_t* active, const float* gate, void* stream);

/* Instructed plasticity, frame-end pieces (BatchInstruct / BatchInstructDeep / BatchInstructDeep2,
 * flyzero/batch.py:226-451); every pointer [device], float32 state updated in place.
 * fb_trace_rates: trace[b][k] += a_pre * (counts[b][upre[k]] * scale_pre - trace[b][k]) and
 *   rate[b][k] += a_rate * (counts[b][upost[k]] * hz - rate[b][k])  (batch.py:282-287). */
int fb_trace_rates(const fb_brain* brain, const int32_t* counts, const int32_t* upre, int32_t n_upre, float* trace,
                   float a_pre, float scale_pre, const int32_t* upost, int32_t n_upost, float* rate, float a_rate,
                   float hz, void* stream);

/* fb_delta_apply: for the plastic entries sel[s] (s < n_sel), per fly f (slots
 * fly_slots[fly_ptr[f] .. fly_ptr[f+1])): d = sum over its slots of coef[b] * trace[b][pre_k[s]] *
 * x[b][post_x[s]], then every slot of the fly w = sign * clip(sign * (w + d), 0, wmax) on the
 * engine's pw (the per-fly averaged delta rule, batch.py:158-172, 312-314, and the fused
 * deep_update kernel, batch.py:26-51). */
int fb_delta_apply(fb_brain* brain, const int32_t* sel, const int32_t* pre_k, const int32_t* post_x, int32_t n_sel,
                   const float* trace, int32_t n_tr, const float* x, int32_t n_x, const float* coef,
                   const int32_t* fly_ptr, const int32_t* fly_slots, int32_t n_flies, const float* sign,
                   const float* wmax, void* stream);

/* fb_backprop: delta[b][pre_l[s]] += (pw[b][sel[s]] / w_syn) * x[b][post_x[s]] (the retrograde
 * error through the fly's own synapses, batch.py:390-393, 440-442; float atomics). */
int fb_backprop(const fb_brain* brain, const int32_t* sel, const int32_t* pre_l, const int32_t* post_x, int32_t n_sel,
                const float* x, int32_t n_x, float* delta, int32_t n_delta, void* stream);

/* Motion-vision front end (MotionEye, flyzero/vision.py:64-191) for every instance, writing the
 * eye neurons' Poisson probabilities straight into p_ext. Parameters as MotionParams
 * (vision.py:34-50): a_hp = float32(1 / tau_hp), a_d = float32(1 / tau_delay), p_scale =
 * float32(dt / 1000); chromatic_gain > 0 computes the blue / green channels, sustained_gain != 0
 * the centre-surround contrast. kernels: 0 = one block per instance when the grid fits in shared
 * memory (else four grid-wide kernels), 1 = one block per instance (FB_ERR_ARG if it does not fit),
 * 2 = the four grid-wide kernels. */
typedef struct fb_eye_params {
    int32_t cell, shift, surround, kernels;
    float a_hp, a_d, p_scale;
    double gain, max_rate, transient_gain, sustained_gain, chromatic_gain;
} fb_eye_params;

/* Floats of eye state for `batch` instances and H x W frames (-1 for a bad geometry). */
int64_t fb_eye_state_floats(int32_t batch, int32_t H, int32_t W, int32_t cell);

/* One frame per instance (MotionEye.see, vision.py:142-191). frames [device] (batch, H, W, 3)
 * uint8; state [device] fb_eye_state_floats floats, kept between frames; restart [device] (batch)
 * uint8: nonzero starts that instance's filters from this frame (the first frame), cleared by the
 * call; flip [device] (batch) uint8 mirrors the frame left-right (flyzero/pool.py:44), or NULL.
 * Per eye neuron [device]: grid column gx, row gy, channel chan (0-7 motion: polarity ON 0 / OFF 1
 * times 4 plus screen direction right 0, left 1, down 2, up 3; 8/9 ON/OFF transient, 10/11 ON/OFF
 * sustained, 12 blue, 13 green), visible (0 above y_min), ext slot. Writes
 * p_ext[b][slot] = float32(max_rate * clip(gain * rate, 0, 1)) * p_scale and, unless NULL,
 * rates [device] (batch, n_cells) in Hz. Ext slots of other neurons are left as they are. */
int fb_motion_eye(fb_brain* brain, const uint8_t* frames, int32_t H, int32_t W, const fb_eye_params* params,
                  float* state, uint8_t* restart, const uint8_t* flip, int32_t n_cells, const int32_t* gx,
                  const int32_t* gy, const uint8_t* chan, const uint8_t* visible, const int32_t* slot, float* rates,
                  void* stream);

/* Choose the schedule (FB_ENGINE_*, FB_PROP_*, lanes per work item 8/16/32; 0 keeps a field). */
int fb_set_schedule(fb_brain* brain, int32_t engine, int32_t propagation, int32_t lanes);

/* Phase trace of the persistent engine (diagnostics). `trace` [device] holds `capacity` int64;
 * every later fb_run whose steps * ctas * 11 fits records, per step and CTA, the SM clock at
 * these points, in step order: 0 step start (accumulator slice requested), 4 next step's kicks
 * drawn, 1 waiting for the slice, 2 slice staged, 3 neurons advanced; 8 listing warps done; per
 * epoch of steps between grid barriers, at its first step 7 push warps start and 10 push warps
 * done, at its last step 5 grid-barrier arrival and 6 grid-barrier exit. NULL: off. No
 * counterpart in the reference. */
int fb_set_trace(fb_brain* brain, long long* trace, int64_t capacity);

/* Limits for fault drills (diagnostics; no counterpart in the reference, whose only guard is a
 * capacity assert, flyzero/gpu.py:166-168). barrier_cycles: the persistent engine's grid-barrier
 * wait budget in SM clock cycles before it gives up, raises FB_ERR_TIMEOUT (fb_check) and every CTA
 * returns (0: the default, about 4 s). item_capacity: work items per spike list, at most the
 * allocated capacity fb_get_info reports; a smaller one makes an active run raise FB_ERR_OVERFLOW
 * (items beyond it are dropped, never written out of bounds; 0: the allocated capacity). The list
 * layout depends on it: change it only right after fb_reset of every instance. A run that timed
 * out or overflowed leaves the simulation invalid: fb_reset it. */
int fb_set_limits(fb_brain* brain, int64_t barrier_cycles, int64_t item_capacity);

/* Device error flags raised since the last call (overflow, barrier timeout), then cleared.
 * Synchronises `stream`. Returns FB_OK or the first raised FB_ERR_* code. */
int fb_check(fb_brain* brain, void* stream);

/* ---------------------------------------------------------------------------------------------
 * Run without any allocation by the library. (This entry point has no counterpart in the
 * reference: it serves callers that cannot allocate device memory at run time, e.g. a program
 * whose GPU memory is owned entirely by another allocator's pool, a control loop that cannot take
 * the device synchronisation a cudaMalloc/cudaFree implies, or a deployment that forbids run-time
 * allocation after start-up.)
 *
 * One instance, every buffer caller-owned and on the device: the CSR exactly as the reference
 * keeps it on the GPU (indptr int64 n+1, indices int32, weights float32 already x w_syn, like
 * flyzero/gpu.py:157-159 with no plastic entries), the state v, g (float32 n) and ref (int8 n),
 * optional ext inputs (ext_idx int32 n, p_ext and bias_ext float32 n_ext; ext_idx NULL = none),
 * and counts (int32 n, overwritten). Poisson kicks use the counter hash with `seed`, `step_no`
 * (first step) and tick t0 (first step), like fb_run. The result equals fb_run of an engine
 * created with FB_FLAG_ACC_FIXED, bit for bit.
 *
 * Its only scratch, the synaptic input in flight, lives in an array compiled into the library:
 * FB_STATIC_RING_ENTRIES int64 (8 MiB), present on every GPU that loads the library until the
 * process exits. A network fits if n * (n_delay + 1) <= FB_STATIC_RING_ENTRIES; larger ones are
 * rejected with FB_ERR_ARG. The array is shared by every call and keeps what the last call left:
 * clear != 0 zeroes the in-flight input first (start of a simulation); clear == 0 continues the
 * previous call's simulation. Calls that overlap on the GPU (other streams, other threads) race
 * on the array. The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress); make that first call before any stream capture. A device reset
 * (cudaDeviceReset) may move the array: the address looked up before it is stale afterwards, so do
 * not call this entry point again in a process that reset the device. t0 must be >= 0, and
 * delay/dt, t_ref/dt finite and at most 1e6 (else FB_ERR_ARG before any device work). No
 * cudaMalloc, cudaFree or allocating library routine is called. */
#define FB_STATIC_RING_ENTRIES 1048576
int fb_run_static(const fb_params* params, int64_t n, const int64_t* indptr, const int32_t* indices,
                  const float* weights, float* v, float* g, int8_t* ref, const int32_t* ext_idx,
                  const float* p_ext, const float* bias_ext, uint32_t seed, uint32_t step_no, int64_t t0,
                  int32_t steps, int32_t clear, int32_t* counts, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FLYBRAIN_H */
