// Motion-vision front end on the device (flyzero/vision.py:142-191, MotionEye.see) for every
// instance at once, writing the eye neurons' Poisson probabilities straight into p_ext: the
// frames are already on the device, so no rates cross the bus and no host loop runs per frame.
//
//   k_eye_cells    one thread per (instance, grid cell):
//                  lum = mean over the cell x cell block of mean(R, G, B) / 255 (vision.py:136-140),
//                  each block row summed with NumPy's pairwise rule, the row sums added in order;
//                  blue / green grids the same way from one channel (chromatic channels);
//                  high-pass lp += a_hp (lum - lp), hp = lum - lp, sig_on = max(hp, 0),
//                  sig_off = max(-hp, 0). An instance whose restart flag is set starts from this
//                  frame: lp = lum, delay arms 0 (vision.py:145-147).
//   k_eye_integral one block per instance: the integral image of the zero-padded lum grid,
//                  cumsum down the columns then along the rows (vision.py:170), float32.
//   k_eye_rates    one thread per (instance, eye neuron): its channel at its grid cell,
//                  motion = the Hassenstein-Reichardt correlator delayed(A) B - A delayed(B) of its
//                  polarity, B the cell `shift` to the right / below, rectified for its screen
//                  direction (vision.py:151-162); columnar channels as vision.py:164-186 (the
//                  sustained contrast in float64, as NumPy promotes it); 0 above y_min;
//                  p_ext[b][slot] = f32(max_rate * clip(gain * rate, 0, 1)) * p_scale. A neuron
//                  whose cell, channel or slot is out of range is skipped.
//   k_eye_delay    one thread per (instance, polarity, cell): d += a_d (sig - d); clears the
//                  instance's restart flag.
// One rounding per operation in the order NumPy evaluates it, no contraction.
#pragma once
#include "common.cuh"

namespace fb {

enum EyeChannel : uint8_t {
    EYE_ON_RIGHT = 0, EYE_ON_LEFT, EYE_ON_DOWN, EYE_ON_UP,
    EYE_OFF_RIGHT, EYE_OFF_LEFT, EYE_OFF_DOWN, EYE_OFF_UP,
    EYE_ON_TRANSIENT, EYE_OFF_TRANSIENT, EYE_ON_SUSTAINED, EYE_OFF_SUSTAINED, EYE_BLUE, EYE_GREEN,
    EYE_CHANNELS
};

struct EyeArgs {
    int32_t B, H, W, cell, gh, gw, shift, surround, chromatic;
    float a_hp, a_d, gain_f, max_rate, p_scale, transient_f, chromatic_f;
    double gain, sustained;
    const uint8_t* frames;      // (B, H, W, 3)
    const uint8_t* flip;        // (B) mirror the frame left-right, or nullptr
    uint8_t* restart;           // (B) start the filters from this frame; cleared by k_eye_delay
    float* lum;                 // (B, gh, gw)
    float* lp;                  // (B, gh, gw)
    float* sig;                 // (B, 2, gh, gw)  ON, OFF
    float* dly;                 // (B, 2, gh, gw)
    float* col;                 // (B, 2, gh, gw)  blue, green
    float* ii;                  // (B, gh + 1, gw + 1)
    int32_t n_cells;
    const int32_t* gx;          // (n_cells) grid column
    const int32_t* gy;          // (n_cells) grid row
    const uint8_t* chan;        // (n_cells) EyeChannel
    const uint8_t* visible;     // (n_cells) 0 above y_min
    const int32_t* slot;        // (n_cells) ext slot
    float* p_ext;               // (B, n_ext)
    int32_t n_ext;
    float* rates;               // (B, n_cells) rates in Hz, or nullptr
};

// NumPy's pairwise float32 sum of n values with the given stride (sequential below 8, eight
// accumulators up to 128 values, then the tail).
template <typename F>
__device__ __forceinline__ float np_row_sum(int32_t n, F at)
{
    if (n < 8) {
        float r = 0.0f;
        for (int32_t i = 0; i < n; i++) r = __fadd_rn(r, at(i));
        return r;
    }
    float a[8];
#pragma unroll
    for (int32_t j = 0; j < 8; j++) a[j] = at(j);
    int32_t i = 8;
    for (; i < n - n % 8; i += 8)
#pragma unroll
        for (int32_t j = 0; j < 8; j++) a[j] = __fadd_rn(a[j], at(i + j));
    float r = __fadd_rn(__fadd_rn(__fadd_rn(a[0], a[1]), __fadd_rn(a[2], a[3])),
                        __fadd_rn(__fadd_rn(a[4], a[5]), __fadd_rn(a[6], a[7])));
    for (; i < n; i++) r = __fadd_rn(r, at(i));
    return r;
}

__global__ void k_eye_cells(const EyeArgs a)
{
    const int64_t cells = (int64_t)a.gh * a.gw;
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (int64_t)a.B * cells) return;
    const int32_t b = (int32_t)(p / cells);
    const int64_t q = p - (int64_t)b * cells;
    const int32_t y = (int32_t)(q / a.gw), x = (int32_t)(q - (int64_t)y * a.gw);
    const bool fl = a.flip && a.flip[b];
    const uint8_t* fr = a.frames + (int64_t)b * a.H * a.W * 3;
    auto px = [&](int32_t yy, int32_t xx) {
        const int32_t c = x * a.cell + xx;
        return fr + ((int64_t)(y * a.cell + yy) * a.W + (fl ? a.W - 1 - c : c)) * 3;
    };
    float s = 0.0f, sb = 0.0f, sg = 0.0f;
    for (int32_t yy = 0; yy < a.cell; yy++) {
        s = __fadd_rn(s, np_row_sum(a.cell, [&](int32_t xx) {
                          const uint8_t* v = px(yy, xx);
                          const float m = __fdiv_rn(__fadd_rn(__fadd_rn((float)v[0], (float)v[1]), (float)v[2]), 3.0f);
                          return __fdiv_rn(m, 255.0f);
                      }));
        if (a.chromatic) {
            sb = __fadd_rn(sb, np_row_sum(a.cell, [&](int32_t xx) { return __fdiv_rn((float)px(yy, xx)[2], 255.0f); }));
            sg = __fadd_rn(sg, np_row_sum(a.cell, [&](int32_t xx) { return __fdiv_rn((float)px(yy, xx)[1], 255.0f); }));
        }
    }
    const float area = (float)(a.cell * a.cell);
    const float lum = __fdiv_rn(s, area);
    a.lum[p] = lum;
    if (a.chromatic) {
        a.col[((int64_t)b * 2 + 0) * cells + q] = __fdiv_rn(sb, area);
        a.col[((int64_t)b * 2 + 1) * cells + q] = __fdiv_rn(sg, area);
    }
    float lp = a.lp[p];
    if (a.restart[b]) {
        lp = lum;
        a.dly[((int64_t)b * 2 + 0) * cells + q] = 0.0f;
        a.dly[((int64_t)b * 2 + 1) * cells + q] = 0.0f;
    }
    lp = __fadd_rn(lp, __fmul_rn(a.a_hp, __fsub_rn(lum, lp)));
    a.lp[p] = lp;
    const float hp = __fsub_rn(lum, lp);
    a.sig[((int64_t)b * 2 + 0) * cells + q] = fmaxf(hp, 0.0f);
    a.sig[((int64_t)b * 2 + 1) * cells + q] = fmaxf(-hp, 0.0f);
}

// blockDim.x >= max(gw, gh) + 1
__global__ void k_eye_integral(const EyeArgs a)
{
    const int32_t b = blockIdx.x, W1 = a.gw + 1;
    const float* lum = a.lum + (int64_t)b * a.gh * a.gw;
    float* ii = a.ii + (int64_t)b * (a.gh + 1) * W1;
    const int32_t t = threadIdx.x;
    if (t <= a.gw) {                       // column t of the padded grid, down the rows
        float c = 0.0f;
        ii[t] = 0.0f;
        for (int32_t i = 1; i <= a.gh; i++) {
            c = __fadd_rn(c, t == 0 ? 0.0f : lum[(int64_t)(i - 1) * a.gw + t - 1]);
            ii[(int64_t)i * W1 + t] = c;
        }
    }
    __syncthreads();
    if (t <= a.gh) {                       // row t, along the columns
        float* r = ii + (int64_t)t * W1;
        float c = r[0];
        for (int32_t j = 1; j <= a.gw; j++) {
            c = __fadd_rn(c, r[j]);
            r[j] = c;
        }
    }
}

__device__ __forceinline__ float eye_motion(const EyeArgs& a, int32_t b, int32_t pol, int32_t dir, int32_t y, int32_t x)
{
    const int64_t cells = (int64_t)a.gh * a.gw;
    const float* sg = a.sig + ((int64_t)b * 2 + pol) * cells;
    const float* dl = a.dly + ((int64_t)b * 2 + pol) * cells;
    const int32_t s = a.shift;
    float corr = 0.0f;
    const int64_t i0 = (int64_t)y * a.gw + x;
    if (dir < 2) {
        if (x < a.gw - s) corr = __fsub_rn(__fmul_rn(dl[i0], sg[i0 + s]), __fmul_rn(sg[i0], dl[i0 + s]));
    } else if (y < a.gh - s) {
        const int64_t i1 = i0 + (int64_t)s * a.gw;
        corr = __fsub_rn(__fmul_rn(dl[i0], sg[i1]), __fmul_rn(sg[i0], dl[i1]));
    }
    return (dir & 1) ? fmaxf(-corr, 0.0f) : fmaxf(corr, 0.0f);
}

// the centre-minus-surround contrast, float64 after the float32 box sum (vision.py:167-174)
__device__ __forceinline__ double eye_contrast(const EyeArgs& a, int32_t b, int32_t y, int32_t x)
{
    const int32_t W1 = a.gw + 1, r = a.surround;
    const float* ii = a.ii + (int64_t)b * (a.gh + 1) * W1;
    const int32_t y0 = min(max(y - r, 0), a.gh), y1 = min(max(y + r + 1, 0), a.gh);
    const int32_t x0 = min(max(x - r, 0), a.gw), x1 = min(max(x + r + 1, 0), a.gw);
    const float num = __fadd_rn(__fsub_rn(__fsub_rn(ii[(int64_t)y1 * W1 + x1], ii[(int64_t)y0 * W1 + x1]),
                                          ii[(int64_t)y1 * W1 + x0]), ii[(int64_t)y0 * W1 + x0]);
    const double sur = __ddiv_rn((double)num, (double)((int64_t)(y1 - y0) * (x1 - x0)));
    return __dsub_rn((double)a.lum[((int64_t)b * a.gh + y) * a.gw + x], sur);
}

__global__ void k_eye_rates(const EyeArgs a)
{
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (int64_t)a.B * a.n_cells) return;
    const int32_t b = (int32_t)(p / a.n_cells), k = (int32_t)(p - (int64_t)b * a.n_cells);
    const int32_t c = a.chan[k], x = a.gx[k], y = a.gy[k], s = a.slot[k];
    if (x < 0 || x >= a.gw || y < 0 || y >= a.gh || c >= EYE_CHANNELS || s < 0 || s >= a.n_ext) return;
    const int64_t cell = ((int64_t)b * a.gh + y) * a.gw + x, cells = (int64_t)a.gh * a.gw;
    float r = 0.0f;
    if (c < EYE_ON_TRANSIENT) {
        r = eye_motion(a, b, c >> 2, c & 3, y, x);
    } else if (c <= EYE_OFF_TRANSIENT) {
        const float hp = a.sig[((int64_t)b * 2 + (c - EYE_ON_TRANSIENT)) * cells + (cell - (int64_t)b * cells)];
        r = __fdiv_rn(__fmul_rn(a.transient_f, hp), a.gain_f);
    } else if (c <= EYE_OFF_SUSTAINED) {
        if (a.sustained != 0.0) {
            const double con = eye_contrast(a, b, y, x);
            const double m = c == EYE_ON_SUSTAINED ? fmax(con, 0.0) : fmax(-con, 0.0);
            r = __double2float_rn(__ddiv_rn(__dmul_rn(a.sustained, m), a.gain));
        }
    } else if (a.chromatic) {
        const float v = a.col[((int64_t)b * 2 + (c - EYE_BLUE)) * cells + (cell - (int64_t)b * cells)];
        r = __fdiv_rn(__fmul_rn(a.chromatic_f, v), a.gain_f);
    }
    if (!a.visible[k]) r = 0.0f;
    const float rate = __fmul_rn(a.max_rate, fminf(fmaxf(__fmul_rn(a.gain_f, r), 0.0f), 1.0f));
    if (a.rates) a.rates[p] = rate;
    a.p_ext[(int64_t)b * a.n_ext + s] = __fmul_rn(rate, a.p_scale);
}

__global__ void k_eye_delay(const EyeArgs a)
{
    const int64_t cells = (int64_t)a.gh * a.gw;
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (int64_t)a.B * 2 * cells) return;
    a.dly[p] = __fadd_rn(a.dly[p], __fmul_rn(a.a_d, __fsub_rn(a.sig[p], a.dly[p])));
    if (p % (2 * cells) == 0) a.restart[p / (2 * cells)] = 0;
}

// ---- the whole eye of one instance in one block ----------------------------------------------------
// The same operations as the four kernels above, in one launch: block b reads its frame once, keeps
// the grid (luminance, ON/OFF signals, delay arms, colour grids, integral image, float64 contrast)
// in shared memory, writes its eye neurons' probabilities, then its new delay arms.

struct EyeSmem {
    int32_t cells, ii, chrom, sust;
    static constexpr int32_t TAB = 766 + 256;  // pixel luminance by R+G+B, channel quotient by byte
    __host__ __device__ size_t bytes() const
    {
        return (size_t)cells * 8 * sust + (size_t)cells * 4 * (5 + 2 * chrom) + (size_t)ii * 4 * sust + TAB * 4;
    }
};

// A pixel's luminance mean(R, G, B) / 255 depends only on the integer R + G + B (the float sum of
// three bytes is exact), and a channel value / 255 only on its byte: the tables hold those
// quotients, computed with the same correctly rounded divisions, so the per-pixel work is a lookup.
// VEC4: cell 4 and W a multiple of 4, so a cell row is three aligned 32-bit words.
template <bool VEC4>
__device__ __forceinline__ void cell_sums(const EyeArgs& a, const uint8_t* fr, bool fl, int32_t y, int32_t x,
                                          const float* t_lum, const float* t_ch, bool chrom, float& s, float& sb,
                                          float& sg)
{
    s = sb = sg = 0.0f;
    if constexpr (VEC4) {
        const int32_t c0 = fl ? a.W - 4 - 4 * x : 4 * x;
#pragma unroll
        for (int32_t yy = 0; yy < 4; yy++) {
            const uint32_t* w = reinterpret_cast<const uint32_t*>(fr + ((int64_t)(4 * y + yy) * a.W + c0) * 3);
            const uint32_t w0 = __ldg(w), w1 = __ldg(w + 1), w2 = __ldg(w + 2);
            uint32_t ch[12];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                ch[j] = (w0 >> (8 * j)) & 255u;
                ch[4 + j] = (w1 >> (8 * j)) & 255u;
                ch[8 + j] = (w2 >> (8 * j)) & 255u;
            }
            float r = 0.0f, rb = 0.0f, rg = 0.0f;
            auto add = [&](int p) {
                r = __fadd_rn(r, t_lum[ch[3 * p] + ch[3 * p + 1] + ch[3 * p + 2]]);
                if (chrom) {
                    rb = __fadd_rn(rb, t_ch[ch[3 * p + 2]]);
                    rg = __fadd_rn(rg, t_ch[ch[3 * p + 1]]);
                }
            };
            if (fl) {                           // the mirrored frame's pixel xx is this segment's 3 - xx
#pragma unroll
                for (int xx = 0; xx < 4; xx++) add(3 - xx);
            } else {
#pragma unroll
                for (int xx = 0; xx < 4; xx++) add(xx);
            }
            s = __fadd_rn(s, r);
            sb = __fadd_rn(sb, rb);
            sg = __fadd_rn(sg, rg);
        }
    } else {
        auto px = [&](int32_t yy, int32_t xx) {
            const int32_t c = x * a.cell + xx;
            return fr + ((int64_t)(y * a.cell + yy) * a.W + (fl ? a.W - 1 - c : c)) * 3;
        };
        for (int32_t yy = 0; yy < a.cell; yy++) {
            s = __fadd_rn(s, np_row_sum(a.cell, [&](int32_t xx) {
                              const uint8_t* v = px(yy, xx);
                              return t_lum[v[0] + v[1] + v[2]];
                          }));
            if (chrom) {
                sb = __fadd_rn(sb, np_row_sum(a.cell, [&](int32_t xx) { return t_ch[px(yy, xx)[2]]; }));
                sg = __fadd_rn(sg, np_row_sum(a.cell, [&](int32_t xx) { return t_ch[px(yy, xx)[1]]; }));
            }
        }
    }
}

template <bool VEC4>
__global__ void __launch_bounds__(1024) k_eye_fused(const EyeArgs a, const EyeSmem L)
{
    extern __shared__ __align__(16) unsigned char eye_smem[];
    const int32_t b = blockIdx.x, cells = L.cells, W1 = a.gw + 1;
    double* s_con = reinterpret_cast<double*>(eye_smem);
    float* s_lum = reinterpret_cast<float*>(eye_smem + (size_t)cells * 8 * L.sust);
    float* s_sig = s_lum + cells;                 // ON, OFF
    float* s_dly = s_sig + 2 * cells;             // ON, OFF
    float* s_col = s_dly + 2 * cells;             // blue, green (chromatic only)
    float* s_ii = s_col + 2 * cells * L.chrom;    // (gh + 1) x (gw + 1) (sustained only)
    float* t_lum = s_ii + L.ii * L.sust;          // 766 + 256 quotient tables
    float* t_ch = t_lum + 766;
    for (int32_t i = threadIdx.x; i < EyeSmem::TAB; i += blockDim.x) {
        if (i < 766) t_lum[i] = __fdiv_rn(__fdiv_rn((float)i, 3.0f), 255.0f);
        else t_ch[i - 766] = __fdiv_rn((float)(i - 766), 255.0f);
    }
    __syncthreads();
    const bool restart = a.restart[b] != 0, fl = a.flip && a.flip[b];
    const uint8_t* fr = a.frames + (int64_t)b * a.H * a.W * 3;
    const float area = (float)(a.cell * a.cell);
    float* lp_g = a.lp + (int64_t)b * cells;
    float* dly_g = a.dly + (int64_t)b * 2 * cells;
    for (int32_t q = threadIdx.x; q < cells; q += blockDim.x) {
        const int32_t y = q / a.gw, x = q - y * a.gw;
        float s, sb, sg;
        cell_sums<VEC4>(a, fr, fl, y, x, t_lum, t_ch, L.chrom != 0, s, sb, sg);
        const float lum = __fdiv_rn(s, area);
        s_lum[q] = lum;
        if (L.chrom) {
            s_col[q] = __fdiv_rn(sb, area);
            s_col[cells + q] = __fdiv_rn(sg, area);
        }
        float lp = restart ? lum : lp_g[q];
        lp = __fadd_rn(lp, __fmul_rn(a.a_hp, __fsub_rn(lum, lp)));
        lp_g[q] = lp;
        const float hp = __fsub_rn(lum, lp);
        s_sig[q] = fmaxf(hp, 0.0f);
        s_sig[cells + q] = fmaxf(-hp, 0.0f);
        s_dly[q] = restart ? 0.0f : dly_g[q];
        s_dly[cells + q] = restart ? 0.0f : dly_g[cells + q];
    }
    __syncthreads();
    if (L.sust) {
        const int32_t t = threadIdx.x;
        if (t <= a.gw) {                          // padded column t, down the rows
            float c = 0.0f;
            s_ii[t] = 0.0f;
            for (int32_t i = 1; i <= a.gh; i++) {
                c = __fadd_rn(c, t == 0 ? 0.0f : s_lum[(i - 1) * a.gw + t - 1]);
                s_ii[i * W1 + t] = c;
            }
        }
        __syncthreads();
        if (t <= a.gh) {                          // row t, along the columns
            float* r = s_ii + t * W1;
            float c = r[0];
            for (int32_t j = 1; j <= a.gw; j++) {
                c = __fadd_rn(c, r[j]);
                r[j] = c;
            }
        }
        __syncthreads();
        const int32_t rr = a.surround;
        for (int32_t q = threadIdx.x; q < cells; q += blockDim.x) {
            const int32_t y = q / a.gw, x = q - y * a.gw;
            const int32_t y0 = min(max(y - rr, 0), a.gh), y1 = min(max(y + rr + 1, 0), a.gh);
            const int32_t x0 = min(max(x - rr, 0), a.gw), x1 = min(max(x + rr + 1, 0), a.gw);
            const float num = __fadd_rn(__fsub_rn(__fsub_rn(s_ii[y1 * W1 + x1], s_ii[y0 * W1 + x1]), s_ii[y1 * W1 + x0]),
                                        s_ii[y0 * W1 + x0]);
            const double sur = __ddiv_rn((double)num, (double)((int64_t)(y1 - y0) * (x1 - x0)));
            s_con[q] = __dsub_rn((double)s_lum[q], sur);
        }
        __syncthreads();
    }
    for (int32_t k = threadIdx.x; k < a.n_cells; k += blockDim.x) {
        const int32_t c = __ldg(a.chan + k), x = __ldg(a.gx + k), y = __ldg(a.gy + k), s = __ldg(a.slot + k);
        if (x < 0 || x >= a.gw || y < 0 || y >= a.gh || c >= EYE_CHANNELS || s < 0 || s >= a.n_ext) continue;
        const int32_t q = y * a.gw + x;
        float r = 0.0f;
        if (c < EYE_ON_TRANSIENT) {
            const int32_t pol = c >> 2, dir = c & 3, sh = a.shift;
            const float* sg = s_sig + pol * cells;
            const float* dl = s_dly + pol * cells;
            float corr = 0.0f;
            if (dir < 2) {
                if (x < a.gw - sh) corr = __fsub_rn(__fmul_rn(dl[q], sg[q + sh]), __fmul_rn(sg[q], dl[q + sh]));
            } else if (y < a.gh - sh) {
                const int32_t q1 = q + sh * a.gw;
                corr = __fsub_rn(__fmul_rn(dl[q], sg[q1]), __fmul_rn(sg[q], dl[q1]));
            }
            r = (dir & 1) ? fmaxf(-corr, 0.0f) : fmaxf(corr, 0.0f);
        } else if (c <= EYE_OFF_TRANSIENT) {
            r = __fdiv_rn(__fmul_rn(a.transient_f, s_sig[(c - EYE_ON_TRANSIENT) * cells + q]), a.gain_f);
        } else if (c <= EYE_OFF_SUSTAINED) {
            if (L.sust) {
                const double con = s_con[q];
                const double m = c == EYE_ON_SUSTAINED ? fmax(con, 0.0) : fmax(-con, 0.0);
                r = __double2float_rn(__ddiv_rn(__dmul_rn(a.sustained, m), a.gain));
            }
        } else if (L.chrom) {
            r = __fdiv_rn(__fmul_rn(a.chromatic_f, s_col[(c - EYE_BLUE) * cells + q]), a.gain_f);
        }
        if (!__ldg(a.visible + k)) r = 0.0f;
        const float rate = __fmul_rn(a.max_rate, fminf(fmaxf(__fmul_rn(a.gain_f, r), 0.0f), 1.0f));
        if (a.rates) a.rates[(int64_t)b * a.n_cells + k] = rate;
        a.p_ext[(int64_t)b * a.n_ext + s] = __fmul_rn(rate, a.p_scale);
    }
    for (int32_t q = threadIdx.x; q < 2 * cells; q += blockDim.x)
        dly_g[q] = __fadd_rn(s_dly[q], __fmul_rn(a.a_d, __fsub_rn(s_sig[q], s_dly[q])));
    if (threadIdx.x == 0) a.restart[b] = 0;
}

}  // namespace fb
