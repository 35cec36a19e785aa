// The steps on either side of the pursuit, on the GPU (sm_100a): clip
// gathers, robust templates and the clip noise covariance that prepare the
// pursuit's inputs (spikesorting_fullpursuit/full_binary_pursuit.py:299-322),
// duplicate removal after it (analyze_spike_timing.py), the template-sum
// search (c_cython/sort_cython.pyx:333-458), and the Wiener-filter and ZCA
// passes over the voltage (wiener_filter.py, preprocessing.py:104-169).
//
// All of it is memory-bound or latency-bound integer and float work: the
// kernels stream rows once and coalesce along the contiguous axis; the few
// sequential recurrences of the reference (duplicate scans, running sums)
// run one thread per unit or row, many units at once.
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "../../include/fbp_b200.h"
#include "../../include/fbp_prepost.h"
#include "fbp_common.cuh"

namespace fbp {
int set_last_error(int code, const char *msg);
}

namespace {

using fbp::ceil_div;

int fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    return fbp::set_last_error(code, buf);
}

#define PP_LAUNCH_CHECK()                                                                  \
    do {                                                                                   \
        cudaError_t e_ = cudaGetLastError();                                               \
        if (e_ != cudaSuccess)                                                             \
            return fail(FBP_ERR_CUDA, "kernel launch failed at %s:%d: %s", __FILE__,       \
                        __LINE__, cudaGetErrorString(e_));                                 \
    } while (0)
#define PP_CUDA(call)                                                                      \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return fail(FBP_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));     \
    } while (0)

int grid_of(u64 items, int threads, int cap = 148 * 16) {
    u64 b = (items + threads - 1) / threads;
    if (b > (u64)cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

// ------------------------------------------------------------------ clips

template <typename T>
__global__ void k_gather_clips(const T *__restrict__ v, u64 n, const long long *__restrict__ chans, u32 nch,
                               const long long *__restrict__ ev, u32 first, u32 count, int w0, u32 W,
                               T *__restrict__ out) {
    const u64 per = (u64)nch * W, total = (u64)count * per;
    for (u64 q = (u64)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (u64)gridDim.x * blockDim.x) {
        const u64 e = q / per, r = q - e * per;
        const u32 k = (u32)(r / W), i = (u32)(r - (u64)k * W);
        const long long s = ev[first + e] + w0 + i;
        out[q] = v[(u64)chans[k] * n + (u64)s];
    }
}

// ------------------------------------------------------------------ robust templates

// Float order as unsigned keys (negative values reversed); +-0 differ in key
// but compare equal as values.
__device__ __forceinline__ u32 fkey(float f) {
    const u32 b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float kfloat(u32 k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// Products rounded on their own (no contraction into a following add), as
// numpy forms an array of squares before it sums them.
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }

// The key of the k-th smallest (0-based) of m keys, radix select by one warp
// (8-bit digits, histogram `hist` of 256 words in shared memory).
template <class KeyOf>
__device__ u32 warp_select(u32 m, u32 k, KeyOf key_of, u32 *hist) {
    const u32 lane = threadIdx.x & 31;
    u32 prefix = 0, mask = 0;
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (u32 b = lane; b < 256; b += 32) hist[b] = 0;
        __syncwarp();
        for (u32 i = lane; i < m; i += 32) {
            const u32 key = key_of(i);
            if ((key & mask) == prefix) atomicAdd(&hist[(key >> shift) & 255u], 1u);
        }
        __syncwarp();
        u32 c[8], s = 0;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            c[j] = hist[8 * lane + j];
            s += c[j];
        }
        const u32 incl = fbp::warp_incl_scan(s), excl = incl - s;
        const bool mine = k >= excl && k < incl;
        const u32 ball = __ballot_sync(0xffffffffu, mine);
        u32 digit = 0, before = 0;
        if (mine) {
            u32 acc = excl;
#pragma unroll
            for (int j = 0; j < 8; j++) {
                if (k >= acc && k < acc + c[j]) { digit = 8 * lane + j; before = acc; }
                acc += c[j];
            }
        }
        const int src = __ffs(ball) - 1;
        digit = __shfl_sync(0xffffffffu, digit, src);
        before = __shfl_sync(0xffffffffu, before, src);
        k -= before;
        prefix |= digit << shift;
        mask |= 255u << shift;
        __syncwarp();
    }
    return prefix;
}

template <typename T> struct RobustArith;
template <> struct RobustArith<float> {    // numpy float32 arithmetic
    typedef float A;
    static __device__ float half_sum(float a, float b) { return __fmul_rn(__fadd_rn(a, b), 0.5f); }
    static __device__ float mad_scale(float m) { return __fdiv_rn(m, 0.6745f); }
    static __device__ float store(float x) { return x; }
};
template <> struct RobustArith<short> {    // numpy: int16 medians in float64, stored truncated
    typedef double A;
    static __device__ double half_sum(double a, double b) { return (a + b) * 0.5; }
    static __device__ double mad_scale(double m) { return __ddiv_rn(m, 0.6745); }
    static __device__ short store(double x) { return (short)__double2int_rz(x); }
};

// Column values of a unit live contiguously in the transposed clips tr[dim][n_rows].
template <typename T>
__global__ void k_transpose(const T *__restrict__ in, u32 rows, u32 cols, T *__restrict__ out) {
    __shared__ T tile[32][33];
    const u32 tiles_c = ceil_div(cols, 32), tiles_r = ceil_div(rows, 32);
    for (u64 t = blockIdx.x; t < (u64)tiles_c * tiles_r; t += gridDim.x) {
        const u32 tr = (u32)(t / tiles_c), tc = (u32)(t % tiles_c);
        for (u32 y = threadIdx.y; y < 32; y += blockDim.y) {
            const u32 r = tr * 32 + y, c = tc * 32 + threadIdx.x;
            if (r < rows && c < cols) tile[y][threadIdx.x] = in[(u64)r * cols + c];
        }
        __syncthreads();
        for (u32 y = threadIdx.y; y < 32; y += blockDim.y) {
            const u32 c = tc * 32 + y, r = tr * 32 + threadIdx.x;
            if (r < rows && c < cols) out[(u64)c * rows + r] = tile[threadIdx.x][y];
        }
        __syncthreads();
    }
}

// calculate_robust_template (preprocessing.py:639-659), one warp per
// (unit, column): the median and the median absolute deviation by radix
// select; the values strictly within one MAD of the median are a contiguous
// range of ranks, whose median is selected directly.
template <typename T>
__global__ void k_robust_template(const T *__restrict__ tr, u32 n_rows, u32 dim, const u32 *__restrict__ off,
                                  u32 n_units, T *__restrict__ out) {
    typedef RobustArith<T> R;
    typedef typename R::A A;
    __shared__ u32 hist_all[8][256];
    const u32 warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    u32 *hist = hist_all[warp];
    const u64 items = (u64)n_units * dim;
    for (u64 it = (u64)blockIdx.x * 8 + warp; it < items; it += (u64)gridDim.x * 8) {
        const u32 u = (u32)(it / dim), col = (u32)(it % dim);
        const u32 r0 = off[u], m = off[u + 1] - off[u];
        if (m == 0) continue;
        const T *x = tr + (u64)col * n_rows + r0;
        T *dst = out + (u64)u * dim + col;
        if (m == 1) {                                  // np.squeeze(clips): the clip itself
            if (lane == 0) *dst = x[0];
            continue;
        }
        auto xk = [&](u32 i) { return fkey((float)x[i]); };
        auto med_of = [&](u32 a, u32 cnt, auto keyf) -> A {   // median of ranks [a, a + cnt)
            if (cnt & 1u) return (A)kfloat(warp_select(m, a + (cnt - 1) / 2, keyf, hist));
            const A lo = (A)kfloat(warp_select(m, a + cnt / 2 - 1, keyf, hist));
            const A hi = (A)kfloat(warp_select(m, a + cnt / 2, keyf, hist));
            return R::half_sum(lo, hi);
        };
        const A med = med_of(0, m, xk);
        auto dk = [&](u32 i) {
            const A d = (A)x[i] - med;
            return fkey((float)(d < (A)0 ? -d : d));    // exact in float32 for both types
        };
        const A mad = R::mad_scale(med_of(0, m, dk));
        const A lo = med - mad, hi = med + mad;
        u32 nle = 0, nlt = 0;                           // #(x <= lo), #(x < hi)
        for (u32 i = lane; i < m; i += 32) {
            const A v = (A)x[i];
            nle += v <= lo;
            nlt += v < hi;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            nle += __shfl_xor_sync(0xffffffffu, nle, o);
            nlt += __shfl_xor_sync(0xffffffffu, nlt, o);
        }
        A res = med;
        if (nlt > nle) res = med_of(nle, nlt - nle, xk);
        if (lane == 0) *dst = R::store(res);
    }
}

// ------------------------------------------------------------------ clip noise covariance

template <typename T>
__device__ __forceinline__ double resid_of(const T *clips, const T *tmpl, const u32 *row_unit, u64 row, u32 dim,
                                           u32 col) {
    const T a = clips[row * dim + col], b = tmpl[(u64)row_unit[row] * dim + col];
    return (double)(T)(a - b);                      // dtype arithmetic (int16 wraps), then float64
}

template <typename T>
__global__ void k_resid_mean(const T *__restrict__ clips, const T *__restrict__ tmpl, const u32 *__restrict__ row_unit,
                             const long long *__restrict__ rows, u32 n_sel, u32 dim, double *__restrict__ sums) {
    // block: 32 columns x 8 row lanes
    const u32 col = blockIdx.x * 32 + threadIdx.x;
    if (col >= dim) return;
    double s = 0.0;
    for (u32 r = blockIdx.y * blockDim.y + threadIdx.y; r < n_sel; r += gridDim.y * blockDim.y)
        s += resid_of(clips, tmpl, row_unit, (u64)rows[r], dim, col);
    atomicAdd(&sums[col], s);
}

constexpr int kCovThreads = 512, kCovPerThread = 24;   // L * L <= 12288: L <= 110

// Per channel c, sum over the selected rows of (x_i - mean_i)(x_j - mean_j),
// i, j < L; blocks take row ranges and add their partial matrix atomically.
template <typename T>
__global__ void k_resid_cov(const T *__restrict__ clips, const T *__restrict__ tmpl, const u32 *__restrict__ row_unit,
                            const long long *__restrict__ rows, u32 n_sel, u32 C, u32 L, const double *__restrict__ sums,
                            double *__restrict__ cov) {
    extern __shared__ double csm[];                  // [32 rows][L] centred values
    const u32 c = blockIdx.x, dim = C * L;
    const u32 parts = gridDim.y, part = blockIdx.y;
    const u32 r_begin = (u32)((u64)n_sel * part / parts), r_end = (u32)((u64)n_sel * (part + 1) / parts);
    const u32 LL = L * L;
    double acc[kCovPerThread];
#pragma unroll
    for (int q = 0; q < kCovPerThread; q++) acc[q] = 0.0;
    for (u32 r0 = r_begin; r0 < r_end; r0 += 32) {
        const u32 nr = min(32u, r_end - r0);
        for (u32 e = threadIdx.x; e < nr * L; e += blockDim.x) {
            const u32 rr = e / L, i = e % L;
            const u32 col = c * L + i;
            csm[rr * L + i] = resid_of(clips, tmpl, row_unit, (u64)rows[r0 + rr], dim, col) - sums[col] / n_sel;
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < kCovPerThread; q++) {
            const u32 o = threadIdx.x + q * blockDim.x;
            if (o < LL) {
                const u32 i = o / L, j = o % L;
                double a = acc[q];
                for (u32 rr = 0; rr < nr; rr++) a = fma(csm[rr * L + i], csm[rr * L + j], a);
                acc[q] = a;
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int q = 0; q < kCovPerThread; q++) {
        const u32 o = threadIdx.x + q * blockDim.x;
        if (o < LL) atomicAdd(&cov[(u64)c * LL + o], acc[q]);
    }
}

__global__ void k_scale(double *__restrict__ x, u64 n, double f) {
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) x[i] *= f;
}

// ------------------------------------------------------------------ numpy's pairwise sum

// np.add.reduce over a contiguous 1-D array (numpy's pairwise summation:
// below 8 elements a plain loop from 0; up to 128 eight accumulators, then
// ((r0+r1)+(r2+r3))+((r4+r5)+(r6+r7)) and the remainder in order; above,
// the halves split at a multiple of 8 below n/2).  f(i) gives element i.
template <typename A, class F>
__device__ A np_pairwise(u64 i0, u64 n, F f) {
    // explicit stack instead of recursion: leaves (<= 128 elements) are
    // summed in order of their position and combined as the recursion would
    struct Fr { u64 i0, n; int state; A left; };
    Fr st[40];
    int sp = 0;
    st[0] = {i0, n, 0, (A)0};
    A ret = (A)0;
    for (;;) {
        Fr &fr = st[sp];
        if (fr.n <= 128) {
            A res;
            if (fr.n < 8) {
                res = (A)0;
                for (u64 i = 0; i < fr.n; i++) res += f(fr.i0 + i);
            } else {
                A r[8];
#pragma unroll
                for (int j = 0; j < 8; j++) r[j] = f(fr.i0 + j);
                u64 i = 8;
                for (; i < fr.n - (fr.n % 8); i += 8) {
#pragma unroll
                    for (int j = 0; j < 8; j++) r[j] += f(fr.i0 + i + j);
                }
                res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
                for (; i < fr.n; i++) res += f(fr.i0 + i);
            }
            // return res to the parent
            for (;;) {
                if (sp == 0) { ret = res; return ret; }
                sp--;
                Fr &p = st[sp];
                if (p.state == 1) {              // left half done: do the right half
                    p.left = res;
                    p.state = 2;
                    u64 n2 = p.n / 2;
                    n2 -= n2 % 8;
                    st[++sp] = {p.i0 + n2, p.n - n2, 0, (A)0};
                    break;
                }
                res = p.left + res;              // right half done
            }
        } else {
            u64 n2 = fr.n / 2;
            n2 -= n2 % 8;
            fr.state = 1;
            st[++sp] = {fr.i0, n2, 0, (A)0};
        }
    }
}

// ------------------------------------------------------------------ duplicates

// sum((clip - template)**2) of every event, np.sum's pairwise order; the
// event's unit found by binary search of the unit offsets.
template <typename TT, typename A>
__global__ void k_event_sse(const float *__restrict__ clips, const TT *__restrict__ tmpl, u32 dim,
                            const u32 *__restrict__ off, u32 n_units, u32 n_events, double *__restrict__ sse) {
    for (u32 e = blockIdx.x * blockDim.x + threadIdx.x; e < n_events; e += gridDim.x * blockDim.x) {
        u32 lo = 0, hi = n_units;                    // last u with off[u] <= e
        while (hi - lo > 1) {
            const u32 mid = (lo + hi) / 2;
            if (off[mid] <= e) lo = mid; else hi = mid;
        }
        const float *c = clips + (u64)e * dim;
        const TT *t = tmpl + (u64)lo * dim;
        auto f = [&](u64 i) -> A {
            const A d = (A)c[i] - (A)t[i];
            return mul_rn(d, d);
        };
        sse[e] = (double)np_pairwise<A>(0, dim, f);
    }
}

// The scans of analyze_spike_timing.py, one thread per unit (curr/next as
// the reference steps them).
__global__ void k_dup_scan(int mode, const long long *__restrict__ ev, const u8 *__restrict__ bp,
                           const double *__restrict__ sse, const u32 *__restrict__ off, u32 n_units, long long tol,
                           u8 *__restrict__ keep) {
    for (u32 u = blockIdx.x * blockDim.x + threadIdx.x; u < n_units; u += gridDim.x * blockDim.x) {
        const u32 a = off[u], n = off[u + 1] - a;
        for (u32 i = 0; i < n; i++) keep[a + i] = 1;
        u32 cur = 0, nxt = 1;
        while (nxt < n) {
            const u32 ci = a + cur, ni = a + nxt;
            if (ev[ni] - ev[ci] <= tol) {
                if (mode == 0) {                         // remove_binary_pursuit_duplicates :127-152
                    if (bp[ci] && bp[ni]) {
                        if (sse[ci] <= sse[ni]) { keep[ni] = 0; nxt++; }
                        else { keep[ci] = 0; cur = nxt; nxt++; }
                    } else if (bp[ci] && !bp[ni]) {
                        nxt++;
                    } else {
                        cur = nxt; nxt++;
                    }
                } else if (mode == 1) {                  // keep_binary_pursuit_duplicates :92-111
                    if (bp[ci] && !bp[ni]) { keep[ni] = 0; nxt++; }
                    else if (!bp[ci] && bp[ni]) { keep[ci] = 0; cur = nxt; nxt++; }
                    else { cur = nxt; nxt++; }
                } else {                                 // remove_spike_event_duplicates :166-182
                    if (sse[ci] <= sse[ni]) { keep[ni] = 0; nxt++; }
                    else { keep[ci] = 0; cur = nxt; nxt++; }
                }
            } else {
                cur = nxt; nxt++;
            }
        }
    }
}

// np.mean(clips, axis=0) for float32: rows added in order, then / count.
__global__ void k_unit_mean(const float *__restrict__ clips, u32 dim, const u32 *__restrict__ off, u32 n_units,
                            float *__restrict__ out) {
    const u64 items = (u64)n_units * dim;
    for (u64 q = (u64)blockIdx.x * blockDim.x + threadIdx.x; q < items; q += (u64)gridDim.x * blockDim.x) {
        const u32 u = (u32)(q / dim), col = (u32)(q % dim);
        const u32 a = off[u], m = off[u + 1] - a;
        float s = 0.0f;
        for (u32 r = 0; r < m; r++) s = __fadd_rn(s, clips[(u64)(a + r) * dim + col]);
        out[q] = m ? __fdiv_rn(s, (float)m) : __int_as_float(0x7fc00000);
    }
}

// ------------------------------------------------------------------ template-sum search

// One warp per (item, shift1): it scans shift2 in order over its lanes and
// keeps the first strictly smallest residual; the per-shift1 results are
// combined in shift order afterwards.  The residual follows the reference
// element by element: sum = float64(t1 shifted) + float64(t2 shifted);
// (test - sum)**2 summed with numpy's pairwise order.
__device__ __forceinline__ double shifted_tpl(const float *t, u32 L, u32 d, int s) {
    // get_shifted_template: within each channel, value at sample i is the
    // template's sample i - s (0 outside)
    const u32 ch = d / L, i = d - ch * L;
    const int j = (int)i - s;
    return (j >= 0 && j < (int)L) ? (double)t[ch * L + j] : 0.0;
}

__global__ void k_overlap_tpl(const float *__restrict__ T, u32 C, u32 L, int n_pre, int n_post,
                              const u32 *__restrict__ items, u32 n_items, double *__restrict__ part_ss,
                              int *__restrict__ part_s2) {
    const u32 S = (u32)(n_pre + n_post + 1), D = C * L;
    const u32 lane = threadIdx.x & 31;
    const u64 tasks = (u64)n_items * S;
    for (u64 task = ((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5; task < tasks;
         task += ((u64)gridDim.x * blockDim.x) >> 5) {
        const u32 it = (u32)(task / S), s1i = (u32)(task % S);
        const float *x = T + (u64)items[3 * it] * D;
        const float *t1 = T + (u64)items[3 * it + 1] * D;
        const float *t2 = T + (u64)items[3 * it + 2] * D;
        const int s1 = (int)s1i - n_pre;
        double best = __longlong_as_double(0x7ff0000000000000ll);   // inf
        int bs2 = -1;
        for (u32 s2i = lane; s2i < S; s2i += 32) {
            const int s2 = (int)s2i - n_pre;
            auto f = [&](u64 d) -> double {
                const double sum = shifted_tpl(t1, L, (u32)d, s1) + shifted_tpl(t2, L, (u32)d, s2);
                const double r = (double)x[d] - sum;
                return mul_rn(r, r);
            };
            const double ss = np_pairwise<double>(0, D, f);
            if (ss < best) { best = ss; bs2 = (int)s2i; }
        }
        // first strictly smallest over the warp, in shift2 order
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ob = __shfl_xor_sync(0xffffffffu, best, o);
            const int os = __shfl_xor_sync(0xffffffffu, bs2, o);
            if (os >= 0 && (bs2 < 0 || ob < best || (ob == best && os < bs2))) { best = ob; bs2 = os; }
        }
        if (lane == 0) {
            part_ss[task] = best;
            part_s2[task] = bs2;
        }
    }
}

__global__ void k_overlap_tpl_pick(const double *__restrict__ part_ss, const int *__restrict__ part_s2, u32 n_items,
                                   u32 S, int n_pre, double *__restrict__ best_ss, int *__restrict__ best_shift) {
    for (u32 it = blockIdx.x * blockDim.x + threadIdx.x; it < n_items; it += gridDim.x * blockDim.x) {
        double b = __longlong_as_double(0x7ff0000000000000ll);
        int s1b = -1, s2b = -1;
        for (u32 s1 = 0; s1 < S; s1++) {             // shift1 outer, strict <: the first minimum
            const double v = part_ss[(u64)it * S + s1];
            if (part_s2[(u64)it * S + s1] >= 0 && v < b) { b = v; s1b = (int)s1; s2b = part_s2[(u64)it * S + s1]; }
        }
        best_ss[it] = b;
        best_shift[2 * it] = s1b < 0 ? 0 : s1b - n_pre;
        best_shift[2 * it + 1] = s2b < 0 ? 0 : s2b - n_pre;
    }
}

// ------------------------------------------------------------------ Wiener filter

template <typename R>
__global__ void k_power(const R *__restrict__ spec, u64 n, R *__restrict__ p) {
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        const R re = spec[2 * i], im = spec[2 * i + 1];
        p[i] = mul_rn(re, re) + mul_rn(im, im);          // abs2: x.real**2 + x.imag**2
    }
}

// The rolling box-car of wiener_filter.py:40-59, one thread per row, the
// reference's running sums in its order and precision (the spectra's: float32
// for float32 voltage, float64 otherwise; np.sum of the first points is the
// pairwise sum), written to tmp then copied back.
template <typename R>
__global__ void k_smooth(R *__restrict__ P, u64 rows, u64 nb, long long smooth, R *__restrict__ tmp) {
    for (u64 r = (u64)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += (u64)gridDim.x * blockDim.x) {
        R *x = P + r * nb, *o = tmp + r * nb;
        const long long half = smooth / 2;
        long long npts = half < (long long)nb ? half : (long long)nb;
        R run = np_pairwise<R>(0, (u64)npts, [&](u64 i) { return x[i]; });
        for (long long i = 0; i < (long long)nb; i++) {
            if (i + half < (long long)nb) { run += x[i + half]; npts += 1; }
            if (i - half > 0) { run -= x[i - half]; npts -= 1; }
            o[i] = run / (R)npts;
        }
        for (u64 i = 0; i < nb; i++) x[i] = o[i];
    }
}

// spec *= S / (S + N + 1e-9), the filter in the spectra's precision
// (wiener_optimal_filter, :124-129).
template <typename R>
__global__ void k_wiener(R *__restrict__ spec, const R *__restrict__ S, const R *__restrict__ N, u64 n) {
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        const R f = S[i] / ((S[i] + N[i]) + (R)1e-9);
        spec[2 * i] = mul_rn(spec[2 * i], f);
        spec[2 * i + 1] = mul_rn(spec[2 * i + 1], f);
    }
}

// ------------------------------------------------------------------ ZCA

// mask[c][s] = 1 when some |v[c][s + k]| > 0.9 thr[c] for |k| <= cushion
// (np.rint(fftconvolve(|v| > thr, ones(2 cushion + 1), 'same')) > 0): a
// block takes a tile of one channel, prefix-counts the exceedances over the
// tile and its halo (block scan), and reads each window's count.
constexpr u32 kMaskThreads = 256, kMaskTile = 2048;
template <typename T>
__global__ void k_zca_mask(const T *__restrict__ v, u32 C, u64 n, const double *__restrict__ thr, int cushion,
                           u8 *__restrict__ mask) {
    extern __shared__ u32 pre[];                     // [span + 1] prefix counts
    const u64 tiles = (n + kMaskTile - 1) / kMaskTile;
    const u32 span = kMaskTile + 2 * (u32)cushion;
    const u32 per = (span + kMaskThreads - 1) / kMaskThreads;
    for (u64 t = blockIdx.x; t < tiles * C; t += gridDim.x) {
        const u32 c = (u32)(t / tiles);
        const long long s0 = (long long)(t % tiles) * kMaskTile;
        const double th = thr[c] * 0.90;
        const u32 q0 = threadIdx.x * per;
        u32 local = 0;
        for (u32 k = 0; k < per; k++) {
            const u32 q = q0 + k;
            const long long s = s0 - cushion + (long long)q;
            u32 f = 0;
            if (q < span && s >= 0 && s < (long long)n) f = fabs((double)v[(u64)c * n + (u64)s]) > th;
            if (q < span) pre[q + 1] = f;
            local += f;
        }
        const u32 ex = fbp::block_excl_scan(local, nullptr);
        u32 run = ex;
        for (u32 k = 0; k < per; k++) {
            const u32 q = q0 + k;
            if (q < span) { run += pre[q + 1]; pre[q + 1] = run; }
        }
        if (threadIdx.x == 0) pre[0] = 0;
        __syncthreads();
        for (u32 q = threadIdx.x; q < kMaskTile; q += kMaskThreads) {
            const long long s = s0 + q;
            if (s < (long long)n) mask[(u64)c * n + (u64)s] = (pre[q + 2 * cushion + 1] - pre[q]) > 0;
        }
        __syncthreads();
    }
}

// Per channel: count, sum and centred sum of squares of unmasked samples.
template <typename T>
__global__ void k_zca_diag(const T *__restrict__ v, const u8 *__restrict__ mask, u32 C, u64 n,
                           double *__restrict__ cnt, double *__restrict__ sum, int pass, double *__restrict__ ssq) {
    __shared__ double red[2][32];
    for (u32 c = blockIdx.x; c < C; c += gridDim.x) {
        double a = 0.0, b = 0.0;
        const double mu = pass ? sum[c] / cnt[c] : 0.0;
        for (u64 s = threadIdx.x; s < n; s += blockDim.x) {
            if (mask[(u64)c * n + s]) continue;
            const double x = (double)v[(u64)c * n + s];
            if (pass) { a += (x - mu) * (x - mu); } else { a += 1.0; b += x; }
        }
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            b += __shfl_xor_sync(0xffffffffu, b, o);
        }
        if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = a; red[1][threadIdx.x >> 5] = b; }
        __syncthreads();
        if (threadIdx.x == 0) {
            double A = 0, B = 0;
            for (u32 w = 0; w < blockDim.x / 32; w++) { A += red[0][w]; B += red[1][w]; }
            if (pass) ssq[c] = A; else { cnt[c] = A; sum[c] = B; }
        }
        __syncthreads();
    }
}

// Off-diagonal: G[i][j] = sum of v_i v_j and P[i][j] = count over samples
// that neither channel masks; 16x16 channel tiles, samples split over blocks.
template <typename T>
__global__ void k_zca_gram(const T *__restrict__ v, const u8 *__restrict__ mask, u32 C, u64 n, u32 chunk,
                           double *__restrict__ G, double *__restrict__ P) {
    __shared__ double xs[16][65];
    __shared__ double ys[16][65];
    __shared__ u8 mx[16][64], my[16][64];
    const u32 tc = ceil_div(C, 16);
    const u32 ti = blockIdx.x / tc, tj = blockIdx.x % tc;
    if (tj < ti) return;                             // upper triangle of tiles
    const u32 li = threadIdx.x / 16, lj = threadIdx.x % 16;   // 256 threads
    const u32 ci = ti * 16 + li, cj = tj * 16 + lj;
    double g = 0.0, p = 0.0;
    const u64 sb = (u64)blockIdx.y * chunk, se = min(n, sb + chunk);
    for (u64 s0 = sb; s0 < se; s0 += 64) {
        for (u32 q = threadIdx.x; q < 16 * 64; q += blockDim.x) {
            const u32 r = q / 64, k = q % 64;
            const u64 s = s0 + k;
            const u32 a = ti * 16 + r, b = tj * 16 + r;
            const bool in = s < se;
            xs[r][k] = (in && a < C) ? (double)v[(u64)a * n + s] : 0.0;
            mx[r][k] = (in && a < C) ? mask[(u64)a * n + s] : (u8)1;
            ys[r][k] = (in && b < C) ? (double)v[(u64)b * n + s] : 0.0;
            my[r][k] = (in && b < C) ? mask[(u64)b * n + s] : (u8)1;
        }
        __syncthreads();
#pragma unroll 8
        for (u32 k = 0; k < 64; k++) {
            const bool ok = !mx[li][k] && !my[lj][k];
            g += ok ? xs[li][k] * ys[lj][k] : 0.0;
            p += ok ? 1.0 : 0.0;
        }
        __syncthreads();
    }
    if (ci < C && cj < C && cj > ci) {
        atomicAdd(&G[(u64)ci * C + cj], g);
        atomicAdd(&P[(u64)ci * C + cj], p);
    }
}

__global__ void k_zca_sigma(u32 C, const double *__restrict__ G, const double *__restrict__ P,
                            const double *__restrict__ cnt, const double *__restrict__ ssq, double *__restrict__ sigma) {
    for (u32 q = blockIdx.x * blockDim.x + threadIdx.x; q < C * C; q += gridDim.x * blockDim.x) {
        const u32 i = q / C, j = q % C;
        double val;
        if (i == j) val = ssq[i] / (cnt[i] - 1.0);
        else if (i < j) val = G[q] / (P[q] - 1.0);
        else val = G[(u64)j * C + i] / (P[(u64)j * C + i] - 1.0);
        sigma[q] = val;
    }
}

template <typename T> __device__ __forceinline__ T cast_out(double x);
template <> __device__ __forceinline__ float cast_out<float>(double x) { return (float)x; }
template <> __device__ __forceinline__ short cast_out<short>(double x) { return (short)(int)__double2ll_rz(x); }

// out = Z @ v tile by tile: a block computes 32 output channels x 256
// samples, the channel sum in ascending order in float64 (16 channels of
// the voltage staged at a time).
template <typename T>
__global__ void k_zca_apply(const double *__restrict__ Z, const T *__restrict__ v, u32 C, u64 n, T *__restrict__ out) {
    __shared__ double zs[32][17];
    __shared__ double vs[16][256];
    const u32 tio = ceil_div(C, 32);
    const u64 tis = (n + 255) / 256;
    for (u64 t = blockIdx.x; t < tio * tis; t += gridDim.x) {
        const u32 i0 = (u32)(t % tio) * 32;
        const u64 s0 = (t / tio) * 256;
        double acc[32];
#pragma unroll
        for (int k = 0; k < 32; k++) acc[k] = 0.0;
        for (u32 c0 = 0; c0 < C; c0 += 16) {
            for (u32 q = threadIdx.x; q < 32 * 16; q += blockDim.x) {
                const u32 r = q / 16, k = q % 16;
                zs[r][k] = (i0 + r < C && c0 + k < C) ? Z[(u64)(i0 + r) * C + c0 + k] : 0.0;
            }
            for (u32 q = threadIdx.x; q < 16 * 256; q += blockDim.x) {
                const u32 k = q / 256, x = q % 256;
                vs[k][x] = (c0 + k < C && s0 + x < n) ? (double)v[(u64)(c0 + k) * n + s0 + x] : 0.0;
            }
            __syncthreads();
            const u32 kmax = min(16u, C - c0);
            for (u32 k = 0; k < kmax; k++) {
                const double x = vs[k][threadIdx.x];
#pragma unroll
                for (int r = 0; r < 32; r++) acc[r] = fma(zs[r][k], x, acc[r]);
            }
            __syncthreads();
        }
        const u64 s = s0 + threadIdx.x;
        if (s < n) {
#pragma unroll
            for (int r = 0; r < 32; r++)
                if (i0 + r < C) out[(u64)(i0 + r) * n + s] = cast_out<T>(acc[r]);
        }
    }
}

// ------------------------------------------------------------------ separability metrics

// compute_separability_metrics + set_bp_threshold (neuron_separability.py:
// 88-152, 251-261), one block per template: template_SS as numpy's float32
// pairwise sum of the squares (the value the pursuit's -0.5 * SS comes
// from), the same sum in float64, the variance sum_c t_c^T Sigma_c t_c in
// float64, the lower confidence bound and the noise threshold in float64.
__global__ void k_separability(const float *__restrict__ T, u32 K, u32 C, u32 L, const double *__restrict__ cov,
                               double sigma_noise, double sigma_ci, float *__restrict__ ss32,
                               double *__restrict__ ss64, double *__restrict__ var, double *__restrict__ lower_ci,
                               double *__restrict__ thr_raw, double *__restrict__ thr) {
    __shared__ double red[2][32];
    const u32 D = C * L;
    for (u32 k = blockIdx.x; k < K; k += gridDim.x) {
        const float *t = T + (u64)k * D;
        double a = 0.0, b = 0.0;
        for (u32 q = threadIdx.x; q < C * L * L; q += blockDim.x) {
            const u32 c = q / (L * L), ij = q % (L * L), i = ij / L, j = ij % L;
            a += (double)t[c * L + i] * cov[(u64)c * L * L + ij] * (double)t[c * L + j];
        }
        for (u32 q = threadIdx.x; q < D; q += blockDim.x) b += (double)t[q] * (double)t[q];
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            b += __shfl_xor_sync(0xffffffffu, b, o);
        }
        if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = a; red[1][threadIdx.x >> 5] = b; }
        __syncthreads();
        if (threadIdx.x == 0) {
            double v = 0.0, s = 0.0;
            for (u32 w = 0; w < blockDim.x / 32; w++) { v += red[0][w]; s += red[1][w]; }
            const float s32 = np_pairwise<float>(0, D, [&](u64 q) { return mul_rn(t[q], t[q]); });
            // numpy: 0.5 * float32 -> float32; the bounds then in float64
            const float e32 = __fmul_rn(0.5f, s32);
            const double sd = sqrt(v);
            const double ci = (double)e32 - sigma_ci * sd;
            const double tr = -(double)e32 + sigma_noise * sd;
            ss32[k] = s32;
            ss64[k] = s;
            var[k] = v;
            lower_ci[k] = ci;
            thr_raw[k] = tr;
            thr[k] = fmax(fmax(tr, 0.0), ci);
        }
        __syncthreads();
    }
}

}  // namespace

// ================================================================== C ABI

extern "C" {

int fbp_get_clips(const void *voltage, int dtype, uint64_t n, uint32_t C, const int64_t *neighbors,
                  uint32_t nch, const int64_t *events, uint32_t first, uint32_t count, int32_t win0, int32_t win1,
                  void *clips, void *stream) {
    fbp::set_last_error(0, "");
    if (count == 0 || nch == 0) return FBP_OK;
    if (!voltage || !neighbors || !events || !clips || win1 <= win0)
        return fail(FBP_ERR_BAD_ARG, "fbp_get_clips: bad arguments");
    (void)C;
    const u32 W = (u32)(win1 - win0);
    const u64 total = (u64)count * nch * W;
    cudaStream_t st = (cudaStream_t)stream;
    if (dtype == FBP_F32)
        k_gather_clips<float><<<grid_of(total, 256), 256, 0, st>>>((const float *)voltage, n, (const long long *)neighbors,
                                                                   nch, (const long long *)events, first, count, win0,
                                                                   W, (float *)clips);
    else if (dtype == FBP_I16)
        k_gather_clips<short><<<grid_of(total, 256), 256, 0, st>>>((const short *)voltage, n, (const long long *)neighbors,
                                                                   nch, (const long long *)events, first, count, win0,
                                                                   W, (short *)clips);
    else
        return fail(FBP_ERR_BAD_ARG, "fbp_get_clips: dtype must be FBP_F32 or FBP_I16");
    PP_LAUNCH_CHECK();
    return FBP_OK;
}

size_t fbp_robust_scratch_bytes(uint32_t n_rows, uint32_t dim, int dtype) {
    return (size_t)n_rows * dim * (dtype == FBP_I16 ? 2 : 4);
}

int fbp_robust_templates(const void *clips, int dtype, uint32_t n_rows, uint32_t dim, const uint32_t *off,
                         uint32_t n_units, void *templates, void *scratch, size_t scratch_bytes, void *stream) {
    fbp::set_last_error(0, "");
    if (n_units == 0 || dim == 0) return FBP_OK;
    if (!clips || !off || !templates || !scratch)
        return fail(FBP_ERR_BAD_ARG, "fbp_robust_templates: null pointer argument");
    if (dtype != FBP_F32 && dtype != FBP_I16)
        return fail(FBP_ERR_BAD_ARG, "fbp_robust_templates: dtype must be FBP_F32 or FBP_I16");
    if (scratch_bytes < fbp_robust_scratch_bytes(n_rows, dim, dtype))
        return fail(FBP_ERR_BAD_ARG, "fbp_robust_templates: scratch too small");
    cudaStream_t st = (cudaStream_t)stream;
    const u64 tiles = (u64)ceil_div(n_rows, 32) * ceil_div(dim, 32);
    const int tgrid = (int)std::min<u64>(tiles, 148ull * 32);
    const u64 items = (u64)n_units * dim;
    const int rgrid = (int)std::min<u64>((items + 7) / 8, 148ull * 64);
    if (n_rows == 0) return FBP_OK;
    if (dtype == FBP_F32) {
        k_transpose<float><<<tgrid, dim3(32, 8), 0, st>>>((const float *)clips, n_rows, dim, (float *)scratch);
        k_robust_template<float><<<rgrid, 256, 0, st>>>((const float *)scratch, n_rows, dim, off, n_units,
                                                        (float *)templates);
    } else {
        k_transpose<short><<<tgrid, dim3(32, 8), 0, st>>>((const short *)clips, n_rows, dim, (short *)scratch);
        k_robust_template<short><<<rgrid, 256, 0, st>>>((const short *)scratch, n_rows, dim, off, n_units,
                                                        (short *)templates);
    }
    PP_LAUNCH_CHECK();
    return FBP_OK;
}

size_t fbp_noise_cov_scratch_bytes(uint32_t C, uint32_t L) { return (size_t)C * L * sizeof(double); }

int fbp_clip_noise_covariance(const void *clips, int dtype, const uint32_t *row_unit, const void *templates,
                              const int64_t *rows, uint32_t n_sel, uint32_t C, uint32_t L, double *cov,
                              void *scratch, size_t scratch_bytes, void *stream) {
    fbp::set_last_error(0, "");
    if (!clips || !row_unit || !templates || !rows || !cov || !scratch)
        return fail(FBP_ERR_BAD_ARG, "fbp_clip_noise_covariance: null pointer argument");
    if (C == 0 || L == 0 || n_sel == 0) return fail(FBP_ERR_BAD_ARG, "fbp_clip_noise_covariance: empty input");
    if (L * L > (u32)(kCovThreads * kCovPerThread))
        return fail(FBP_ERR_BAD_ARG, "fbp_clip_noise_covariance: L = %u above 110", L);
    if (scratch_bytes < fbp_noise_cov_scratch_bytes(C, L))
        return fail(FBP_ERR_BAD_ARG, "fbp_clip_noise_covariance: scratch too small");
    cudaStream_t st = (cudaStream_t)stream;
    double *sums = (double *)scratch;
    const u32 dim = C * L;
    PP_CUDA(cudaMemsetAsync(sums, 0, (size_t)dim * 8, st));
    PP_CUDA(cudaMemsetAsync(cov, 0, (size_t)C * L * L * 8, st));
    const dim3 mb(32, 8), mg(ceil_div(dim, 32), std::min<u32>(64, ceil_div(n_sel, 8)));
    const u32 parts = std::max<u32>(1, std::min<u32>(ceil_div(n_sel, 256), ceil_div(148 * 4, C)));
    const size_t smem = (size_t)32 * L * sizeof(double);
    if (dtype == FBP_F32) {
        k_resid_mean<float><<<mg, mb, 0, st>>>((const float *)clips, (const float *)templates, row_unit,
                                               (const long long *)rows, n_sel, dim, sums);
        k_resid_cov<float><<<dim3(C, parts), kCovThreads, smem, st>>>((const float *)clips, (const float *)templates, row_unit,
                                                              (const long long *)rows, n_sel, C, L, sums, cov);
    } else if (dtype == FBP_I16) {
        k_resid_mean<short><<<mg, mb, 0, st>>>((const short *)clips, (const short *)templates, row_unit,
                                               (const long long *)rows, n_sel, dim, sums);
        k_resid_cov<short><<<dim3(C, parts), kCovThreads, smem, st>>>((const short *)clips, (const short *)templates, row_unit,
                                                              (const long long *)rows, n_sel, C, L, sums, cov);
    } else {
        return fail(FBP_ERR_BAD_ARG, "fbp_clip_noise_covariance: dtype must be FBP_F32 or FBP_I16");
    }
    k_scale<<<grid_of((u64)C * L * L, 256), 256, 0, st>>>(cov, (u64)C * L * L, 1.0 / (double)n_sel);
    PP_LAUNCH_CHECK();
    return FBP_OK;
}

int fbp_remove_duplicates(int mode, const int64_t *events, const uint8_t *bp_bool, const float *clips,
                          const void *templates, int tdtype, uint32_t dim, const uint32_t *off, uint32_t n_units,
                          uint32_t n_events, int64_t tol, double *sse, uint8_t *keep, void *stream) {
    fbp::set_last_error(0, "");
    if (n_events == 0 || n_units == 0) return FBP_OK;
    if (mode < 0 || mode > 2) return fail(FBP_ERR_BAD_ARG, "fbp_remove_duplicates: mode must be 0, 1 or 2");
    if (!events || !off || !keep || (mode != 2 && !bp_bool) || (mode != 1 && (!clips || !templates || !sse)))
        return fail(FBP_ERR_BAD_ARG, "fbp_remove_duplicates: null pointer argument");
    cudaStream_t st = (cudaStream_t)stream;
    if (mode != 1) {
        if (tdtype == FBP_F32)
            k_event_sse<float, float><<<grid_of(n_events, 128), 128, 0, st>>>(clips, (const float *)templates, dim,
                                                                                off, n_units, n_events, sse);
        else if (tdtype == FBP_F64)
            k_event_sse<double, double><<<grid_of(n_events, 128), 128, 0, st>>>(clips, (const double *)templates, dim,
                                                                                  off, n_units, n_events, sse);
        else
            return fail(FBP_ERR_BAD_ARG, "fbp_remove_duplicates: template dtype must be FBP_F32 or FBP_F64");
    }
    k_dup_scan<<<grid_of(n_units, 64), 64, 0, st>>>(mode, (const long long *)events, bp_bool, sse, off, n_units,
                                                    (long long)tol, keep);
    PP_LAUNCH_CHECK();
    return FBP_OK;
}

int fbp_unit_mean_templates(const float *clips, uint32_t dim, const uint32_t *off, uint32_t n_units,
                            float *templates, void *stream) {
    fbp::set_last_error(0, "");
    if (n_units == 0 || dim == 0) return FBP_OK;
    if (!clips || !off || !templates) return fail(FBP_ERR_BAD_ARG, "fbp_unit_mean_templates: null pointer argument");
    k_unit_mean<<<grid_of((u64)n_units * dim, 256), 256, 0, (cudaStream_t)stream>>>(clips, dim, off, n_units,
                                                                                     templates);
    PP_LAUNCH_CHECK();
    return FBP_OK;
}

size_t fbp_overlap_template_scratch_bytes(uint32_t n_items, int32_t n_pre, int32_t n_post) {
    const size_t S = (size_t)(n_pre + n_post + 1);
    return (size_t)n_items * S * 12;
}

int fbp_overlap_template_search(const float *templates, uint32_t K, uint32_t C, uint32_t L, int32_t n_pre,
                                int32_t n_post, const uint32_t *items, uint32_t n_items, double *best_ss,
                                int32_t *best_shift, void *scratch, size_t scratch_bytes, void *stream) {
    fbp::set_last_error(0, "");
    if (n_items == 0) return FBP_OK;
    if (!templates || !items || !best_ss || !best_shift || !scratch || n_pre < 0 || n_post < 0 || L == 0 || C == 0)
        return fail(FBP_ERR_BAD_ARG, "fbp_overlap_template_search: bad arguments");
    if (scratch_bytes < fbp_overlap_template_scratch_bytes(n_items, n_pre, n_post))
        return fail(FBP_ERR_BAD_ARG, "fbp_overlap_template_search: scratch too small");
    (void)K;
    cudaStream_t st = (cudaStream_t)stream;
    const u32 S = (u32)(n_pre + n_post + 1);
    double *part_ss = (double *)scratch;
    int *part_s2 = (int *)(part_ss + (size_t)n_items * S);
    const u64 warps = (u64)n_items * S;
    k_overlap_tpl<<<grid_of(warps * 32, 256, 148 * 64), 256, 0, st>>>(templates, C, L, n_pre, n_post, items, n_items,
                                                                      part_ss, part_s2);
    k_overlap_tpl_pick<<<grid_of(n_items, 128), 128, 0, st>>>(part_ss, part_s2, n_items, S, n_pre, best_ss,
                                                               best_shift);
    PP_LAUNCH_CHECK();
    return FBP_OK;
}

int fbp_power_spectrum(const void *spec, int dtype, uint64_t rows, uint64_t nb, void *power, void *stream) {
    fbp::set_last_error(0, "");
    if (!spec || !power) return fail(FBP_ERR_BAD_ARG, "fbp_power_spectrum: null pointer argument");
    const u64 n = rows * nb;
    if (n == 0) return FBP_OK;
    cudaStream_t st = (cudaStream_t)stream;
    if (dtype == FBP_F32) k_power<float><<<grid_of(n, 256), 256, 0, st>>>((const float *)spec, n, (float *)power);
    else if (dtype == FBP_F64) k_power<double><<<grid_of(n, 256), 256, 0, st>>>((const double *)spec, n, (double *)power);
    else return fail(FBP_ERR_BAD_ARG, "fbp_power_spectrum: dtype must be FBP_F32 or FBP_F64");
    PP_LAUNCH_CHECK();
    return FBP_OK;
}

int fbp_wiener_smooth(void *power, int dtype, uint64_t rows, uint64_t nb, int64_t smooth, void *scratch,
                      void *stream) {
    fbp::set_last_error(0, "");
    if (smooth <= 1 || rows == 0 || nb == 0) return FBP_OK;
    if (!power || !scratch) return fail(FBP_ERR_BAD_ARG, "fbp_wiener_smooth: null pointer argument");
    cudaStream_t st = (cudaStream_t)stream;
    if (dtype == FBP_F32)
        k_smooth<float><<<grid_of(rows, 32), 32, 0, st>>>((float *)power, rows, nb, (long long)smooth, (float *)scratch);
    else if (dtype == FBP_F64)
        k_smooth<double><<<grid_of(rows, 32), 32, 0, st>>>((double *)power, rows, nb, (long long)smooth,
                                                           (double *)scratch);
    else return fail(FBP_ERR_BAD_ARG, "fbp_wiener_smooth: dtype must be FBP_F32 or FBP_F64");
    PP_LAUNCH_CHECK();
    return FBP_OK;
}

int fbp_wiener_apply(void *spec, const void *S, const void *N, int dtype, uint64_t rows, uint64_t nb, void *stream) {
    fbp::set_last_error(0, "");
    if (!spec || !S || !N) return fail(FBP_ERR_BAD_ARG, "fbp_wiener_apply: null pointer argument");
    const u64 n = rows * nb;
    if (n == 0) return FBP_OK;
    cudaStream_t st = (cudaStream_t)stream;
    if (dtype == FBP_F32)
        k_wiener<float><<<grid_of(n, 256), 256, 0, st>>>((float *)spec, (const float *)S, (const float *)N, n);
    else if (dtype == FBP_F64)
        k_wiener<double><<<grid_of(n, 256), 256, 0, st>>>((double *)spec, (const double *)S, (const double *)N, n);
    else return fail(FBP_ERR_BAD_ARG, "fbp_wiener_apply: dtype must be FBP_F32 or FBP_F64");
    PP_LAUNCH_CHECK();
    return FBP_OK;
}

size_t fbp_zca_scratch_bytes(uint32_t C) { return ((size_t)2 * C * C + 3 * (size_t)C) * sizeof(double); }

int fbp_zca_covariance(const void *voltage, int dtype, uint32_t C, uint64_t n, const double *thr, int32_t cushion,
                       uint8_t *mask, double *sigma, void *scratch, size_t scratch_bytes, void *stream) {
    fbp::set_last_error(0, "");
    if (!voltage || !thr || !mask || !sigma || !scratch)
        return fail(FBP_ERR_BAD_ARG, "fbp_zca_covariance: null pointer argument");
    if (C == 0 || n == 0 || cushion < 0) return fail(FBP_ERR_BAD_ARG, "fbp_zca_covariance: bad sizes");
    if (scratch_bytes < fbp_zca_scratch_bytes(C)) return fail(FBP_ERR_BAD_ARG, "fbp_zca_covariance: scratch too small");
    cudaStream_t st = (cudaStream_t)stream;
    double *G = (double *)scratch, *P = G + (size_t)C * C, *cnt = P + (size_t)C * C, *sum = cnt + C, *ssq = sum + C;
    PP_CUDA(cudaMemsetAsync(G, 0, (size_t)2 * C * C * 8, st));
    const u32 mthreads = kMaskThreads;
    const size_t msmem = ((size_t)kMaskTile + 2 * (size_t)cushion + 2) * 4;
    if (msmem > 200 * 1024) return fail(FBP_ERR_BAD_ARG, "fbp_zca_covariance: cushion too large");
    const u64 mtiles = (n + kMaskTile - 1) / kMaskTile * C;
    const u32 tcs = ceil_div(C, 16);
    const u32 chunk = 1u << 16;
    const dim3 gg(tcs * tcs, (u32)((n + chunk - 1) / chunk));
    if (dtype == FBP_F32) {
        const float *v = (const float *)voltage;
        if (msmem > 48 * 1024) PP_CUDA(cudaFuncSetAttribute(k_zca_mask<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)msmem));
        k_zca_mask<float><<<(int)std::min<u64>(mtiles, 148 * 8), mthreads, msmem, st>>>(v, C, n, thr, cushion, mask);
        k_zca_diag<float><<<std::min<u32>(C, 148 * 4), 256, 0, st>>>(v, mask, C, n, cnt, sum, 0, ssq);
        k_zca_diag<float><<<std::min<u32>(C, 148 * 4), 256, 0, st>>>(v, mask, C, n, cnt, sum, 1, ssq);
        k_zca_gram<float><<<gg, 256, 0, st>>>(v, mask, C, n, chunk, G, P);
    } else if (dtype == FBP_I16) {
        const short *v = (const short *)voltage;
        if (msmem > 48 * 1024) PP_CUDA(cudaFuncSetAttribute(k_zca_mask<short>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)msmem));
        k_zca_mask<short><<<(int)std::min<u64>(mtiles, 148 * 8), mthreads, msmem, st>>>(v, C, n, thr, cushion, mask);
        k_zca_diag<short><<<std::min<u32>(C, 148 * 4), 256, 0, st>>>(v, mask, C, n, cnt, sum, 0, ssq);
        k_zca_diag<short><<<std::min<u32>(C, 148 * 4), 256, 0, st>>>(v, mask, C, n, cnt, sum, 1, ssq);
        k_zca_gram<short><<<gg, 256, 0, st>>>(v, mask, C, n, chunk, G, P);
    } else {
        return fail(FBP_ERR_BAD_ARG, "fbp_zca_covariance: dtype must be FBP_F32 or FBP_I16");
    }
    k_zca_sigma<<<grid_of((u64)C * C, 256), 256, 0, st>>>(C, G, P, cnt, ssq, sigma);
    PP_LAUNCH_CHECK();
    return FBP_OK;
}

int fbp_zca_apply(const double *zca, const void *voltage, int dtype, uint32_t C, uint64_t n, void *out, void *stream) {
    fbp::set_last_error(0, "");
    if (!zca || !voltage || !out) return fail(FBP_ERR_BAD_ARG, "fbp_zca_apply: null pointer argument");
    if (C == 0 || n == 0) return FBP_OK;
    cudaStream_t st = (cudaStream_t)stream;
    const u64 tiles = (u64)ceil_div(C, 32) * ((n + 255) / 256);
    const int grid = (int)std::min<u64>(tiles, 148ull * 4);
    if (dtype == FBP_F32) {
        k_zca_apply<float><<<grid, 256, 0, st>>>(zca, (const float *)voltage, C, n, (float *)out);
    } else if (dtype == FBP_I16) {
        k_zca_apply<short><<<grid, 256, 0, st>>>(zca, (const short *)voltage, C, n, (short *)out);
    } else {
        return fail(FBP_ERR_BAD_ARG, "fbp_zca_apply: dtype must be FBP_F32 or FBP_I16");
    }
    PP_LAUNCH_CHECK();
    return FBP_OK;
}

int fbp_separability_metrics(const float *templates, uint32_t K, uint32_t C, uint32_t L, const double *cov,
                             double sigma_noise, double sigma_ci, float *ss32, double *ss64, double *var,
                             double *lower_ci, double *thr_raw, double *thr, void *stream) {
    fbp::set_last_error(0, "");
    if (K == 0) return FBP_OK;
    if (!templates || !cov || !ss32 || !ss64 || !var || !lower_ci || !thr_raw || !thr || C == 0 || L == 0)
        return fail(FBP_ERR_BAD_ARG, "fbp_separability_metrics: bad arguments");
    k_separability<<<std::min<u32>(K, 148 * 8), 256, 0, (cudaStream_t)stream>>>(
        templates, K, C, L, cov, sigma_noise, sigma_ci, ss32, ss64, var, lower_ci, thr_raw, thr);
    PP_LAUNCH_CHECK();
    return FBP_OK;
}

}  // extern "C"
