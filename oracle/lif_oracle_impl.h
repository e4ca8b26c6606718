/* Body of the oracle, instantiated once per state precision by lif_oracle.c
 * (REAL = float or double, SFX = f32 or f64). Test infrastructure only. */

/* ------------------------------------------------------------------------------------------
 * The reference step, statement for statement: flyzero/brain.py:32-58 (`_kernel`).
 *   pass 1 (brain.py:39-45): g = g*decay_syn + buf; buf = 0; refractory decrement or Euler v;
 *   pass 2 (brain.py:46-48): Poisson kicks, input entry by input entry;
 *   pass 3 (brain.py:49-56): threshold, reset, count, push of the CSR row into the same slot.
 * Synaptic input is summed in REAL, one CSR entry at a time in spike order, exactly as the
 * reference does. `contract` != 0 fuses g*decay_syn + buf and v + e*decay_m into single-rounding
 * FMAs: the only transformation the shipped kernel's fastmath (brain.py:62) applies to this code
 * (its `contract` flag alone reproduces it bit for bit; `reassoc` changes nothing).
 * Kicks come from a precomputed raster over input entries:
 * bit j of row s  <=>  `np.random.random() < p_in[j]` at step s of the reference stream.
 * ------------------------------------------------------------------------------------------ */
int64_t CAT(fbo_ref_run_, SFX)(int64_t steps, int64_t t, int32_t n_delay, int64_t n,
                               REAL* restrict v, REAL* restrict g, int16_t* restrict ref,
                               REAL* restrict pending, int32_t* restrict counts,
                               const int64_t* indptr, const int32_t* indices, const REAL* data,
                               const int64_t* input_idx, int64_t n_in, const uint32_t* kicks,
                               REAL kick, REAL decay_syn, REAL decay_m, REAL v_rest, REAL v_th,
                               REAL v_reset, int16_t n_ref, const REAL* restrict bias, int32_t contract,
                               int32_t* step_counts, uint64_t* step_digest)
{
    const int64_t words = (n_in + 31) / 32;
    for (int64_t s = 0; s < steps; s++) {
        REAL* restrict buf = pending + (t % n_delay) * n;
        /* pass 1, if-converted so that it vectorises: the membrane value is computed for every
         * neuron and kept only where the neuron is not refractory (same per-element operations). */
        if (contract) {
            for (int64_t i = 0; i < n; i++) {
                const REAL gi = FMA(g[i], decay_syn, buf[i]);
                g[i] = gi;
                buf[i] = 0;
                const int16_t r = ref[i];
                const REAL vo = v[i];
                const REAL e = gi + bias[i] - (vo - v_rest);
                const REAL vn = FMA(e, decay_m, vo);
                v[i] = r > 0 ? vo : vn;
                ref[i] = (int16_t)(r - (r > 0));
            }
        } else {
            for (int64_t i = 0; i < n; i++) {
                const REAL gi = g[i] * decay_syn + buf[i];
                g[i] = gi;
                buf[i] = 0;
                const int16_t r = ref[i];
                const REAL vo = v[i];
                const REAL e = gi + bias[i] - (vo - v_rest);
                const REAL vn = vo + e * decay_m;
                v[i] = r > 0 ? vo : vn;
                ref[i] = (int16_t)(r - (r > 0));
            }
        }
        if (kicks) {
            const uint32_t* row = kicks + s * words;
            for (int64_t j = 0; j < n_in; j++)
                if ((row[j >> 5] >> (j & 31)) & 1u) v[input_idx[j]] += kick;
        }
        int32_t nsp = 0;
        uint64_t dig = 0;
        for (int64_t i = 0; i < n; i++) {
            if (v[i] >= v_th && ref[i] <= 0) {
                v[i] = v_reset;
                ref[i] = n_ref;
                counts[i] += 1;
                nsp++;
                dig += fbo_spike_tag((uint64_t)i);
                for (int64_t k = indptr[i]; k < indptr[i + 1]; k++) buf[indices[k]] += data[k];
            }
        }
        if (step_counts) step_counts[s] = nsp;
        if (step_digest) step_digest[s] = dig;
        t += 1;
    }
    return t;
}

/* ------------------------------------------------------------------------------------------
 * The engine's batched semantics: B instances share the CSR; each has its own state, outside
 * input ("ext" slots, flyzero/gpu.py:174-179, 201-226) and plastic weights (gpu.py:150-163).
 * Order of operations per instance-neuron is the reference's (brain.py:39-56, gpu.py:48-84).
 * Differences from the reference, all deliberate and shared bit-for-bit with the CUDA engine:
 *   - synaptic input accumulates exactly: INT32 signed synapse counts (acc_mode 0, scaled once:
 *     buf = (REAL)isum * w_syn) or INT64 Q32.32 fixed point for arbitrary float weights
 *     (acc_mode 1: buf = (REAL)(isum * 2^-32));
 *   - plastic entries keep their connectome weight in the fixed part; each instance's float32
 *     weight pw enters as a Q32.32 delta over it, q32(pw) - q32(w0), pushed at spike time and
 *     added after the fixed part: buf = buf + (REAL)(psum * 2^-32) (so pw == w0 adds exactly 0);
 *   - Poisson kicks come from a raster over ext slots (parity) or from the counter hash of the
 *     reference GPU engine (gpu.py:29-31, 63-69): h = mix(tid ^ mix(step*phi ^ mix(seed + b))).
 * All REAL arithmetic is written as separate IEEE operations (this file is compiled with
 * -ffp-contract=off), except the two products that net->contract fuses exactly where the
 * shipped reference kernel fuses them (numba fastmath = LLVM `contract`: g*decay_syn + buf and
 * v + e*decay_m); no reassociation.
 * Instance b advances at tick t only while t < stop_tick[b] (stop_tick NULL: always).
 * ------------------------------------------------------------------------------------------ */
int64_t CAT(fbo_engine_run_, SFX)(const fbo_net* net, int64_t steps, int64_t t, uint32_t step_no,
                                  REAL* v, REAL* g, int8_t* ref, void* ring, int64_t* pring,
                                  int32_t* counts, const float* pw, const int32_t* ext_idx,
                                  int32_t n_ext, const float* p_ext, const float* bias_ext,
                                  const uint32_t* kicks, uint32_t seed, const int64_t* stop_tick,
                                  int32_t* step_counts, uint64_t* step_digest)
{
    const int64_t n = net->n, B = net->B;
    const int32_t nd = net->n_delay;
    const REAL ds = (REAL)net->CAT(decay_syn_, SFX), dm = (REAL)net->CAT(decay_m_, SFX);
    const REAL kick = (REAL)net->CAT(kick_, SFX), wsyn = (REAL)net->CAT(w_syn_, SFX);
    const REAL v_rest = (REAL)net->CAT(v_rest_, SFX), v_th = (REAL)net->CAT(v_th_, SFX);
    const REAL v_reset = (REAL)net->CAT(v_reset_, SFX);
    const int64_t words = (n_ext + 31) / 32;
    int32_t* ring32 = (int32_t*)ring;
    int64_t* ring64 = (int64_t*)ring;
    for (int64_t s = 0; s < steps; s++, t++, step_no++) {
        const int64_t slot = t % nd;
        for (int64_t b = 0; b < B; b++) {
            if (stop_tick && t >= stop_tick[b]) {
                if (step_counts) step_counts[s * B + b] = 0;
                if (step_digest) step_digest[s * B + b] = 0;
                continue;
            }
            REAL* vb = v + b * n;
            REAL* gb = g + b * n;
            int8_t* rb = ref + b * n;
            const int64_t base = (slot * B + b) * n;
            /* pass 1: arriving input, decay, membrane */
            for (int64_t i = 0; i < n; i++) {
                REAL buf;
                if (net->acc_mode == 0) {
                    int32_t x = ring32[base + i];
                    ring32[base + i] = 0;
                    buf = (REAL)x * wsyn;
                } else {
                    int64_t x = ring64[base + i];
                    ring64[base + i] = 0;
                    buf = (REAL)((double)x * FBO_Q32_INV);
                }
                if (pring && net->is_ppost[i]) {
                    int64_t x = pring[base + i];
                    pring[base + i] = 0;
                    buf = buf + (REAL)((double)x * FBO_Q32_INV);
                }
                REAL gi = net->contract ? FMA(gb[i], ds, buf) : gb[i] * ds + buf;
                gb[i] = gi;
                const int32_t j = ext_idx ? ext_idx[i] : -1;
                if (rb[i] > 0) {
                    rb[i] -= 1;
                } else {
                    REAL a = (j >= 0) ? gi + (REAL)bias_ext[b * n_ext + j] : gi;
                    REAL d = vb[i] - v_rest;
                    REAL e = a - d;
                    vb[i] = net->contract ? FMA(e, dm, vb[i]) : vb[i] + e * dm;
                }
                /* pass 2 (per neuron: a kick only touches its own neuron) */
                if (j >= 0) {
                    int hit;
                    if (kicks) {
                        const uint32_t w = kicks[(s * B + b) * words + (j >> 5)];
                        hit = (int)((w >> (j & 31)) & 1u);
                    } else {
                        const float p = p_ext[b * n_ext + j];
                        hit = 0;
                        if (p > 0.0f) {
                            uint32_t tid = (uint32_t)(b * n + i);
                            uint32_t h = fbo_mix32(tid ^ fbo_mix32(step_no * 0x9e3779b9u ^ fbo_mix32(seed + (uint32_t)b)));
                            hit = ((float)(h >> 8) * (1.0f / 16777216.0f)) < p;
                        }
                    }
                    if (hit) vb[i] = vb[i] + kick;
                }
            }
            /* pass 3: threshold, reset, push into the slot just read (arrives n_delay later) */
            int32_t nsp = 0;
            uint64_t dig = 0;
            for (int64_t i = 0; i < n; i++) {
                if (vb[i] >= v_th && rb[i] <= 0) {
                    vb[i] = v_reset;
                    rb[i] = (int8_t)net->n_ref;
                    counts[b * n + i] += 1;
                    nsp++;
                    dig += fbo_spike_tag((uint64_t)i);
                    for (int64_t k = net->indptr[i]; k < net->indptr[i + 1]; k++) {
                        if (net->acc_mode == 0) ring32[base + net->indices[k]] += net->cnt[k];
                        else ring64[base + net->indices[k]] += net->wfx[k];
                    }
                    if (pring) {
                        for (int64_t k = net->pl_indptr[i]; k < net->pl_indptr[i + 1]; k++)
                            pring[base + net->pl_post[k]] += fbo_q32(pw[b * net->n_pl + k]) - net->pl_q0[k];
                    }
                }
            }
            if (step_counts) step_counts[s * B + b] = nsp;
            if (step_digest) step_digest[s * B + b] = dig;
        }
    }
    return t;
}
