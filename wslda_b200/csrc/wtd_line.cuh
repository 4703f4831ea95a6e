/*
 * Register-resident FFT of one lattice line (the 3D path's building block).
 *
 * line_fwd/line_inv: a thread owns one whole line of n points (one x-, y- or z-line of one
 * field) in a register array C v[n]; team_fwd/team_inv below split a line over T threads.  The forward transform is decimation in frequency (natural order in,
 * digit-reversed order out), the inverse runs the exact reverse stages (digit-reversed in,
 * natural out), unnormalised, with cuFFT's sign conventions — the transform the shared-memory
 * FFT of wtd_core.cuh computes, here with every loop fully unrolled so that each index is a
 * compile-time constant: the line stays in registers, the twiddle reads are immediate-offset
 * loads of a shared-memory table, and twiddles that are powers of -i become swaps and sign
 * changes.  k-space multipliers address the digit-reversed position p of frequency
 * dif_freq(n, p), a compile-time constant too.
 *
 * Radices: 8, 4, 2, 3 by the hand-written butterflies of wtd_core.cuh; any other prime by the
 * direct DFT over the line's twiddle table (tw[t] = e^{-2 pi i t/n}, n entries).
 */
#ifndef WTD_LINE_CUH
#define WTD_LINE_CUH

#include "wtd_core.cuh"

/* Table and coefficient reads that do not change while a kernel runs would be hoisted out of
 * the kernels' state loops and kept in registers (hundreds of them).  The kernels therefore
 * read them through a base pointer made opaque once per loop iteration: inside the iteration
 * the loads are ordinary (scheduled and batched freely), across iterations they are issued
 * again. */
template <typename T> __device__ __forceinline__ T *opaque_ptr(T *p)
{
    asm volatile("" : "+l"(p));
    return p;
}
template <typename T> __device__ __forceinline__ T lds_tab(const T *p) { return *p; }

/* a * e^{-2 pi i t/n} (SIGN < 0) or a * e^{+2 pi i t/n} (SIGN > 0); t folds to a constant
 * inside the unrolled stages, and so do the branches */
/* tw: the table of the full line, n * ST entries (ST = the stride of a sub-line of n points
 * inside a line of n * ST points) */
template <int n, int SIGN, int ST, typename C>
__device__ __forceinline__ C line_twiddle(C a, const C *tw, int t)
{
    t %= n;
    if (t == 0) return a;
    if (4 * t == n) return mul_i<SIGN>(a);            /* (-i)^1 or i^1 */
    if (2 * t == n) { C r; r.x = -a.x; r.y = -a.y; return r; }
    if (4 * t == 3 * n) return mul_i<-SIGN>(a);
    const C w = lds_tab(tw + t * ST);
    return SIGN < 0 ? cmul(a, w) : cmulc(a, w);
}

/* forward stages of sub-transform length L (down to 1) */
template <int n, int L, int ST, typename C>
__device__ __forceinline__ void line_fwd_stages(C (&v)[n], const C *tw)
{
    if constexpr (L > 1) {
        constexpr int R = radix_first(L), m = L / R, twmul = n / L;
#pragma unroll
        for (int s = 0; s < n / L; s++) {
#pragma unroll
            for (int j = 0; j < m; j++) {
                C a[R];
#pragma unroll
                for (int q = 0; q < R; q++) a[q] = v[s * L + j + q * m];
                dft_r<-1, R>(a, tw, (n / R) * ST);
#pragma unroll
                for (int q = 1; q < R; q++) a[q] = line_twiddle<n, -1, ST>(a[q], tw, j * q * twmul);
#pragma unroll
                for (int q = 0; q < R; q++) v[s * L + j + q * m] = a[q];
            }
        }
        line_fwd_stages<n, L / R, ST>(v, tw);
    }
}

/* inverse stages: the innermost (shortest) stage first, then outward */
template <int n, int L, int ST, typename C>
__device__ __forceinline__ void line_inv_stages(C (&v)[n], const C *tw)
{
    if constexpr (L > 1) {
        constexpr int R = radix_first(L), m = L / R, twmul = n / L;
        line_inv_stages<n, L / R, ST>(v, tw);
#pragma unroll
        for (int s = 0; s < n / L; s++) {
#pragma unroll
            for (int j = 0; j < m; j++) {
                C a[R];
#pragma unroll
                for (int q = 0; q < R; q++) a[q] = v[s * L + j + q * m];
#pragma unroll
                for (int q = 1; q < R; q++) a[q] = line_twiddle<n, +1, ST>(a[q], tw, j * q * twmul);
                dft_r<+1, R>(a, tw, (n / R) * ST);
#pragma unroll
                for (int q = 0; q < R; q++) v[s * L + j + q * m] = a[q];
            }
        }
    }
}

template <int n, int ST = 1, typename C> __device__ __forceinline__ void line_fwd(C (&v)[n], const C *tw) { line_fwd_stages<n, n, ST>(v, tw); }
template <int n, int ST = 1, typename C> __device__ __forceinline__ void line_inv(C (&v)[n], const C *tw) { line_inv_stages<n, n, ST>(v, tw); }

/* ---------------------------------------------------------------------------------------
 * Team transform: T threads (consecutive lanes of one warp) share a line of n points,
 * n = T * n1 with T | n1.  Thread g holds the slice x = g + T i (i < n1) in v[i].
 *   forward: n1-point transforms of the slices (line_fwd, twiddle stride T), twiddles
 *            w_n^{g k1}, exchange through the line's scratch (T rows of n1 + 1), and T-point
 *            transforms across the slices: thread g ends with X[k1 + n1 k2] for
 *            k1 = g S + s (S = n1 / T) and every k2, in v[s T + k2];
 *   inverse: the exact reverse, unnormalised.
 * The frequency of register r of thread g is team_k<n, T>(g, r), in natural order, so the
 * multiplier tables are natural-order tables.  With T = 1 this is line_fwd/line_inv with the
 * digit-reversed frequencies dif_freq(n, r).
 * -------------------------------------------------------------------------------------*/
/* complex numbers of the scratch of one line of n points shared by T threads (T rows of
 * n/T + 1, padded against bank conflicts) */
__host__ __device__ constexpr int team_scratch(int n, int T) { return T > 1 ? T * (n / T + 1) : 0; }

template <int n, int T> struct Team {
    static_assert(T == 1 || T == 2 || T == 4, "team of 1, 2 or 4 threads");
    static_assert(n % (T * T) == 0, "T^2 must divide the line length");
    static constexpr int n1 = n / T;
    static constexpr int S = n1 / T;
    static constexpr int pitch = n1 + 1;
    static constexpr int scratch = team_scratch(n, T);     /* complex numbers of a line's scratch */
};

template <int n, int T>
__device__ __forceinline__ int team_k(int g, int r)
{
    if constexpr (T == 1) return dif_freq(n, r);
    else return g * Team<n, T>::S + r / T + Team<n, T>::n1 * (r % T);
}

template <int n, int T, typename C>
__device__ __forceinline__ void team_fwd(C (&v)[n / T], C *scr, int g, const C *tw)
{
    constexpr int n1 = Team<n, T>::n1, S = Team<n, T>::S, P = Team<n, T>::pitch;
    line_fwd<n1, T>(v, tw);
    if constexpr (T > 1) {
        __syncwarp();
#pragma unroll
        for (int p = 0; p < n1; p++) {
            const int k1 = dif_freq(n1, p);
            scr[g * P + k1] = cmul(v[p], lds_tab(tw + g * k1));
        }
        __syncwarp();
#pragma unroll
        for (int s = 0; s < S; s++) {
            C a[T];
#pragma unroll
            for (int h = 0; h < T; h++) a[h] = scr[h * P + g * S + s];
            dft_r<-1, T>(a, tw, n / T);
#pragma unroll
            for (int k2 = 0; k2 < T; k2++) v[s * T + k2] = a[k2];
        }
    }
}

template <int n, int T, typename C>
__device__ __forceinline__ void team_inv(C (&v)[n / T], C *scr, int g, const C *tw)
{
    constexpr int n1 = Team<n, T>::n1, S = Team<n, T>::S, P = Team<n, T>::pitch;
    if constexpr (T > 1) {
        __syncwarp();
#pragma unroll
        for (int s = 0; s < S; s++) {
            C a[T];
#pragma unroll
            for (int k2 = 0; k2 < T; k2++) a[k2] = v[s * T + k2];
            dft_r<+1, T>(a, tw, n / T);
#pragma unroll
            for (int h = 0; h < T; h++) scr[h * P + g * S + s] = a[h];
        }
        __syncwarp();
#pragma unroll
        for (int p = 0; p < n1; p++) {
            const int k1 = dif_freq(n1, p);
            v[p] = cmulc(scr[g * P + k1], lds_tab(tw + g * k1));
        }
    }
    line_inv<n1, T>(v, tw);
}

/* k-space operators on a team-transformed line, with natural-order multiplier tables of the
 * axis prepared once per CTA (line_tables):
 *   team_mul_lap: v *= lapk[k] = -k^2 / n
 *   team_mul_d:   v *= i dk[k],  dk[k] = k / n with the Nyquist mode zeroed
 *                 (the reference's derivative multipliers, pca_derivative.cu:152-171) */
template <int n, int T, typename C, typename R>
__device__ __forceinline__ void team_mul_lap(C (&v)[n / T], const R *lapk, int g)
{
#pragma unroll
    for (int r = 0; r < n / T; r++) {
        const R s = lds_tab(lapk + team_k<n, T>(g, r));
        v[r].x *= s;
        v[r].y *= s;
    }
}
template <int n, int T, typename C, typename R>
__device__ __forceinline__ void team_mul_d(C (&v)[n / T], const R *dk, int g)
{
#pragma unroll
    for (int r = 0; r < n / T; r++) {
        const R s = lds_tab(dk + team_k<n, T>(g, r));
        C t; t.x = -s * v[r].y; t.y = s * v[r].x;
        v[r] = t;
    }
}

/* per-axis tables of the line transforms in shared memory: twiddles e^{-2 pi i t/n_a} and the
 * two multipliers of natural-order frequencies, in the compute precision */
template <typename TC, int NMAX> struct LineTab {
    typedef typename cplx<TC>::t C;
    C tw[3][NMAX];
    TC lapk[3][NMAX];
    TC dk[3][NMAX];
};

/* fill from the lattice tables: gtw (axes back to back, offsets 0, NX, NX+NY) and gk (rows 0-2
 * wave numbers of digit-reversed positions, rows 3-5 with the Nyquist mode zeroed, ktstride
 * entries per row): position p holds frequency dif_freq(n_a, p) */
template <typename TC, int NMAX, int N0, int N1, int N2>
__device__ __forceinline__ void line_tables(LineTab<TC, NMAX> &t, const double2 *gtw, const double *gk, int ktstride)
{
    const int nax[3] = {N0, N1, N2}, off[3] = {0, N0, N0 + N1};
    for (int i = threadIdx.x; i < 3 * NMAX; i += blockDim.x) {
        const int a = i / NMAX, p = i - a * NMAX;
        const int na = nax[a];
        if (p < na) {
            const double2 w = gtw[off[a] + p];
            t.tw[a][p].x = (TC)w.x;
            t.tw[a][p].y = (TC)w.y;
            const int k = dif_freq(na, p);
            const double kv = gk[a * ktstride + p], kn = gk[(3 + a) * ktstride + p];
            t.lapk[a][k] = (TC)(-(kv * kv) / (double)na);
            t.dk[a][k] = (TC)(kn / (double)na);
        }
    }
}

#endif
