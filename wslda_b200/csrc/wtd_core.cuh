/*
 * Device building blocks of the B200 TD step: complex arithmetic on double2/float2, the
 * in-shared-memory mixed-radix FFT used for the spectral kinetic and gradient terms, and
 * CTA reductions.
 *
 * FFT design.  A lattice field lives in shared memory in natural (x-slowest) order with one
 * pad element every 8 elements of the fastest axis, so that the stride-8 butterflies of the
 * last radix-8 stage hit distinct banks.  The forward transform is decimation in frequency
 * (natural in -> digit-reversed out); the inverse is the exact reverse sequence of stages
 * (digit-reversed in -> natural out), so no reordering pass exists.  k-space operations
 * (multiply by i*k_d or -|k|^2) look the wave number of a digit-reversed position up in a
 * small per-axis table.  Sign conventions follow cuFFT: forward e^{-2 pi i k n/N}, inverse
 * e^{+2 pi i k n/N}, unnormalised; the 1/N of the reference's derivative kernels
 * (hpc-engine/pca_derivative.cu:163-166) is folded into the k-space multiplier.
 *
 * Radices 8, 4, 2 and 3 have hand-written butterflies; any other prime factor p of an axis
 * (5, 7, 11, ... — the reference accepts every even extent, wslda_predefines_test.h:10-36)
 * takes a direct p-point DFT whose roots of unity are read from the axis twiddle table
 * (w_p^m = w_n^{m n/p}), so every even lattice size transforms exactly as with cuFFT.
 */
#ifndef WTD_CORE_CUH
#define WTD_CORE_CUH

#include <cuda_runtime.h>
#include <stdint.h>


/* ---------------------------------------------------------------------------------------
 * complex helpers
 * -------------------------------------------------------------------------------------*/
template <typename T> struct cplx;
template <> struct cplx<double> { typedef double2 t; };
template <> struct cplx<float> { typedef float2 t; };

__device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }
__device__ __forceinline__ float2 mk(float a, float b) { return make_float2(a, b); }
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { C r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { C r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
template <typename C> __device__ __forceinline__ C cmul(C a, C b)
{
    C r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
/* a * conj(b) */
template <typename C> __device__ __forceinline__ C cmulc(C a, C b)
{
    C r; r.x = a.x * b.x + a.y * b.y; r.y = a.y * b.x - a.x * b.y; return r;
}
template <typename C, typename R> __device__ __forceinline__ C cscale(C a, R s) { C r; r.x = a.x * s; r.y = a.y * s; return r; }
/* multiply by -i (forward) or +i (inverse) */
template <int SIGN, typename C> __device__ __forceinline__ C mul_i(C a)
{
    C r;
    if (SIGN < 0) { r.x = a.y; r.y = -a.x; } else { r.x = -a.y; r.y = a.x; }
    return r;
}
__device__ __forceinline__ double2 to_d(float2 a) { return make_double2((double)a.x, (double)a.y); }
__device__ __forceinline__ double2 to_d(double2 a) { return a; }
template <typename C> __device__ __forceinline__ C from_d(double2 a);
template <> __device__ __forceinline__ double2 from_d<double2>(double2 a) { return a; }
template <> __device__ __forceinline__ float2 from_d<float2>(double2 a) { return make_float2((float)a.x, (float)a.y); }

/* ---------------------------------------------------------------------------------------
 * Compile-time lattice geometry.  N0 is the slowest axis (x); absent axes have extent 1.
 * Padded layout: one pad element per 8 elements along the fastest axis.
 * -------------------------------------------------------------------------------------*/
__host__ __device__ constexpr int pad_index(int fast_index) { return fast_index + (fast_index >> 3); }

__host__ __device__ constexpr int smallest_odd_factor(int n, int p = 3) { return (p * p > n) ? n : (n % p == 0 ? p : smallest_odd_factor(n, p + 2)); }
__host__ __device__ constexpr int radix_first(int n) { return (n % 8 == 0) ? 8 : (n % 4 == 0) ? 4 : (n % 2 == 0) ? 2 : smallest_odd_factor(n); }
__host__ __device__ constexpr int radix_at(int n, int s) { return s == 0 ? radix_first(n) : radix_at(n / radix_first(n), s - 1); }
__host__ __device__ constexpr int n_stages(int n) { return n <= 1 ? 0 : 1 + n_stages(n / radix_first(n)); }
/* wave-number index of the digit-reversed output position p of an n-point DIF transform */
__host__ __device__ constexpr int dif_freq(int n, int p)
{
    /* p = k1*(n/r1) + k2*(n/(r1 r2)) + ...; frequency = k1 + r1*k2 + r1*r2*k3 + ... */
    int f = 0, place = 1, len = n;
    while (len > 1) {
        int r = radix_first(len);
        int m = len / r;
        int k = p / m;
        p -= k * m;
        f += k * place;
        place *= r;
        len = m;
    }
    return f;
}

template <int N0_, int N1_, int N2_> struct Geo {
    static constexpr int N0 = N0_, N1 = N1_, N2 = N2_;
    static constexpr int dims = (N2 > 1) ? 3 : (N1 > 1) ? 2 : 1;
    static constexpr int ntot = N0 * N1 * N2;
    static constexpr int nfast = (dims == 3) ? N2 : (dims == 2) ? N1 : N0;
    static constexpr int pitch = pad_index(nfast - 1) + 1;      /* padded row length */
    static constexpr int rows = ntot / nfast;
    static constexpr int padded = rows * pitch;                 /* padded field size */
    static constexpr int n(int a) { return a == 0 ? N0 : a == 1 ? N1 : N2; }
    /* padded offset of natural linear index i */
    __host__ __device__ static constexpr int off(int i) { return (i / nfast) * pitch + pad_index(i % nfast); }
    /* twiddle table: per axis n entries, axes back to back */
    static constexpr int twoff(int a) { return a == 0 ? 0 : a == 1 ? N0 : N0 + N1; }
    static constexpr int twtotal = N0 + N1 + N2;
};

/* ---------------------------------------------------------------------------------------
 * r-point DFT kernels (in registers).  SIGN=-1 forward, +1 inverse.
 * -------------------------------------------------------------------------------------*/
template <int SIGN, typename C> __device__ __forceinline__ void dft2(C *a)
{
    C t = a[0]; a[0] = cadd(t, a[1]); a[1] = csub(t, a[1]);
}
template <int SIGN, typename C> __device__ __forceinline__ void dft4(C *a)
{
    C s0 = cadd(a[0], a[2]), d0 = csub(a[0], a[2]);
    C s1 = cadd(a[1], a[3]), d1 = mul_i<SIGN>(csub(a[1], a[3]));
    a[0] = cadd(s0, s1); a[2] = csub(s0, s1);
    a[1] = cadd(d0, d1); a[3] = csub(d0, d1);
}
template <int SIGN, typename C> __device__ __forceinline__ void dft3(C *a)
{
    typedef decltype(a[0].x) R;
    const R h = (R)0.86602540378443864676; /* sin(2 pi/3) */
    C s = cadd(a[1], a[2]), d = csub(a[1], a[2]);
    C m; m.x = a[0].x - (R)0.5 * s.x; m.y = a[0].y - (R)0.5 * s.y;
    C w = mul_i<SIGN>(cscale(d, h));
    a[0] = cadd(a[0], s);
    a[1] = cadd(m, w);
    a[2] = csub(m, w);
}
template <int SIGN, typename C> __device__ __forceinline__ void dft8(C *a)
{
    typedef decltype(a[0].x) R;
    const R r2 = (R)0.70710678118654752440; /* 1/sqrt(2) */
    /* radix-2 first layer: pairs (q, q+4) */
    C b[8];
#pragma unroll
    for (int q = 0; q < 4; q++) { b[q] = cadd(a[q], a[q + 4]); b[q + 4] = csub(a[q], a[q + 4]); }
    /* twiddles w8^q on the difference half */
    {
        C t = b[5]; /* * e^{SIGN i pi/4} */
        b[5].x = r2 * (t.x - (R)SIGN * t.y); b[5].y = r2 * (t.y + (R)SIGN * t.x);
        b[6] = mul_i<SIGN>(b[6]);
        t = b[7]; /* * e^{SIGN i 3pi/4} */
        b[7].x = r2 * (-t.x - (R)SIGN * t.y); b[7].y = r2 * (-t.y + (R)SIGN * t.x);
    }
    C e[4] = {b[0], b[1], b[2], b[3]}, o[4] = {b[4], b[5], b[6], b[7]};
    dft4<SIGN>(e);
    dft4<SIGN>(o);
    a[0] = e[0]; a[2] = e[1]; a[4] = e[2]; a[6] = e[3];
    a[1] = o[0]; a[3] = o[1]; a[5] = o[2]; a[7] = o[3];
}
/* direct R-point DFT for any other (prime) radix: X_k = sum_q x_q w_R^{SIGN' qk}, the roots
 * taken from the axis table tw[t] = e^{-2 pi i t/n} at t = (qk mod R) * (n/R) */
template <int SIGN, int R, typename C> __device__ __forceinline__ void dft_gen(C *a, const C *tw, int nR)
{
    C out[R];
#pragma unroll
    for (int k = 0; k < R; k++) {
        C acc = a[0];
#pragma unroll
        for (int q = 1; q < R; q++) {
            const C w = tw[((q * k) % R) * nR];
            acc = cadd(acc, SIGN < 0 ? cmul(a[q], w) : cmulc(a[q], w));
        }
        out[k] = acc;
    }
#pragma unroll
    for (int k = 0; k < R; k++) a[k] = out[k];
}
template <int SIGN, int R, typename C> __device__ __forceinline__ void dft_r(C *a, const C *tw, int nR)
{
    if constexpr (R == 8) dft8<SIGN>(a);
    else if constexpr (R == 4) dft4<SIGN>(a);
    else if constexpr (R == 2) dft2<SIGN>(a);
    else if constexpr (R == 3) dft3<SIGN>(a);
    else dft_gen<SIGN, R>(a, tw, nR);
}

/* ---------------------------------------------------------------------------------------
 * One radix-R stage (sub-transform length L) over every line of axis AX, all threads of the
 * CTA.  buf: padded field in smem; tw: e^{-2 pi i t/n} for this axis (n entries).
 * Forward (SIGN=-1): DIF butterfly then twiddle w_L^{jq}.  Inverse (SIGN=+1): multiply by
 * conj(w_L^{jq}), then the inverse butterfly — the exact reverse of the forward stage.
 * -------------------------------------------------------------------------------------*/
template <class G, int AX, int L, int R, int SIGN, int NF, typename C>
__device__ __forceinline__ void fft_stage(C *buf, int fstride, const C *tw)
{
    constexpr int n = G::n(AX);
    constexpr int m = L / R;
    constexpr int nbfly = G::ntot / R;
    constexpr int twmul = n / L;
    constexpr bool fast = (AX == G::dims - 1);
    constexpr int st = fast ? 1 : (AX == 0 ? (G::ntot / G::N0 / G::nfast) * G::pitch : G::pitch);
    for (int b = threadIdx.x; b < nbfly; b += blockDim.x) {
        int j, s, lineoff;
        if (fast) {
            constexpr int per_line = n / R;
            int line = b / per_line, w = b - line * per_line;
            s = w / m; j = w - s * m;
            lineoff = line * G::pitch;
        } else {
            constexpr int others = G::ntot / n;
            int o = b % others, w = b / others;
            s = w / m; j = w - s * m;
            if (G::dims == 2) {                       /* AX == 0, o = y */
                lineoff = pad_index(o);
            } else if (AX == 0) {                     /* o = (y, z) */
                int y = o / G::N2, z = o - y * G::N2;
                lineoff = y * G::pitch + pad_index(z);
            } else {                                  /* AX == 1, o = (x, z) */
                int x = o / G::N2, z = o - x * G::N2;
                lineoff = x * G::N1 * G::pitch + pad_index(z);
            }
        }
        const int base = s * L + j;
        int addr[R];
#pragma unroll
        for (int q = 0; q < R; q++) {
            int e = base + q * m;
            addr[q] = fast ? lineoff + pad_index(e) : lineoff + e * st;
        }
        C v[NF][R];
#pragma unroll
        for (int f = 0; f < NF; f++)
#pragma unroll
            for (int q = 0; q < R; q++) v[f][q] = buf[f * fstride + addr[q]];
        C w[R];
#pragma unroll
        for (int q = 1; q < R; q++) w[q] = tw[(j * q * twmul) % n];
#pragma unroll
        for (int f = 0; f < NF; f++) {
            if (SIGN > 0) {
#pragma unroll
                for (int q = 1; q < R; q++) v[f][q] = cmulc(v[f][q], w[q]);
                dft_r<SIGN, R>(v[f], tw, n / R);
            } else {
                dft_r<SIGN, R>(v[f], tw, n / R);
#pragma unroll
                for (int q = 1; q < R; q++) v[f][q] = cmul(v[f][q], w[q]);
            }
        }
#pragma unroll
        for (int f = 0; f < NF; f++)
#pragma unroll
            for (int q = 0; q < R; q++) buf[f * fstride + addr[q]] = v[f][q];
    }
}

/* forward stages of axis AX from stage S on (sub-transform length L); NF fields */
template <class G, int AX, int S, int L, int NF, typename C>
__device__ __forceinline__ void fft_axis_fwd(C *buf, int fstride, const C *tw)
{
    if constexpr (L > 1) {
        constexpr int R = radix_first(L);
        fft_stage<G, AX, L, R, -1, NF>(buf, fstride, tw);
        __syncthreads();
        fft_axis_fwd<G, AX, S + 1, L / R, NF>(buf, fstride, tw);
    }
}
/* inverse stages of axis AX: recurse to the innermost stage first, then undo outward */
template <class G, int AX, int L, int NF, typename C>
__device__ __forceinline__ void fft_axis_inv(C *buf, int fstride, const C *tw)
{
    if constexpr (L > 1) {
        constexpr int R = radix_first(L);
        fft_axis_inv<G, AX, L / R, NF>(buf, fstride, tw);
        fft_stage<G, AX, L, R, +1, NF>(buf, fstride, tw);
        __syncthreads();
    }
}

/* forward transform of NF fields (natural -> digit reversed) */
template <class G, int NF, typename C>
__device__ __forceinline__ void fft_forward(C *buf, int fstride, const C *twtab)
{
    fft_axis_fwd<G, 0, 0, G::N0, NF>(buf, fstride, twtab + G::twoff(0));
    if constexpr (G::dims >= 2) fft_axis_fwd<G, 1, 0, G::N1, NF>(buf, fstride, twtab + G::twoff(1));
    if constexpr (G::dims >= 3) fft_axis_fwd<G, 2, 0, G::N2, NF>(buf, fstride, twtab + G::twoff(2));
}

/* inverse transform of NF fields (digit reversed -> natural), unnormalised */
template <class G, int NF, typename C>
__device__ __forceinline__ void fft_inverse(C *buf, int fstride, const C *twtab)
{
    if constexpr (G::dims >= 3) fft_axis_inv<G, 2, G::N2, NF>(buf, fstride, twtab + G::twoff(2));
    if constexpr (G::dims >= 2) fft_axis_inv<G, 1, G::N1, NF>(buf, fstride, twtab + G::twoff(1));
    fft_axis_inv<G, 0, G::N0, NF>(buf, fstride, twtab + G::twoff(0));
}

/* ---------------------------------------------------------------------------------------
 * asynchronous L2 prefetch of a contiguous range (sm_90+ bulk prefetch, no registers or
 * shared memory used; completion is not tracked — later ordinary loads simply hit L2).
 * addr and bytes must be multiples of 16.
 * -------------------------------------------------------------------------------------*/
__device__ __forceinline__ void prefetch_l2(const void *addr, size_t bytes)
{
    const char *p = (const char *)addr;
    while (bytes > 0) {
        unsigned chunk = bytes > 32768 ? 32768u : (unsigned)bytes;
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(chunk) : "memory");
        p += chunk;
        bytes -= chunk;
    }
}

/* L2 residency policies (createpolicy): data reused across states — the per-CTA density
 * slots and the per-point H coefficients — is kept (evict_last) while the state stream passes
 * through (evict_first / .cs) */
__device__ __forceinline__ uint64_t l2_policy_keep()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ double ld_keep(const double *a, uint64_t pol)
{
    double v;
    asm volatile("ld.global.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(a), "l"(pol));
    return v;
}
/* read-only load with the same L2 policy, not volatile: for arrays that no thread writes while
 * the kernel runs, so the compiler may schedule and batch these loads freely */
__device__ __forceinline__ double ld_ro_keep(const double *a, uint64_t pol)
{
    double v;
    asm("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(a), "l"(pol));
    return v;
}
__device__ __forceinline__ void st_keep(double *a, double v, uint64_t pol)
{
    asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(a), "d"(v), "l"(pol) : "memory");
}
/* *a += v as a reduction performed in L2 (no value returned, so the thread does not wait for
 * it), with the same policy.  Used where every address of a slot is updated by one thread
 * only: reductions of one thread to one address take effect in program order, so the sum's
 * order, and therefore its rounding, is that of a plain read-modify-write loop. */
__device__ __forceinline__ void red_keep(double *a, double v, uint64_t pol)
{
    asm volatile("red.relaxed.gpu.global.add.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(a), "d"(v), "l"(pol) : "memory");
}

/* streaming loads/stores (evict-first): state and history arrays are touched once per pass */
__device__ __forceinline__ double2 ld_stream(const double2 *p) { return __ldcs(p); }
__device__ __forceinline__ float2 ld_stream(const float2 *p) { return __ldcs(p); }
__device__ __forceinline__ void st_stream(double2 *p, double2 v) { __stcs(p, v); }
__device__ __forceinline__ void st_stream(float2 *p, float2 v) { __stcs(p, v); }

/* ---------------------------------------------------------------------------------------
 * reductions
 * -------------------------------------------------------------------------------------*/
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

/* sum over the CTA; red must hold >= 32 doubles; result broadcast to every thread */
__device__ __forceinline__ double block_sum(double v, double *red)
{
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    double s = 0.0;
    if (wid == 0) {
        s = (lane < nw) ? red[lane] : 0.0;
        s = warp_sum(s);
        if (lane == 0) red[32] = s;
    }
    __syncthreads();
    return red[32];
}

/* two sums at once */
__device__ __forceinline__ double2 block_sum2(double a, double b, double *red)
{
    a = warp_sum(a); b = warp_sum(b);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if (lane == 0) { red[wid] = a; red[32 + wid] = b; }
    __syncthreads();
    if (wid == 0) {
        double s = (lane < nw) ? red[lane] : 0.0, t = (lane < nw) ? red[32 + lane] : 0.0;
        s = warp_sum(s); t = warp_sum(t);
        if (lane == 0) { red[64] = s; red[65] = t; }
    }
    __syncthreads();
    return make_double2(red[64], red[65]);
}

#endif
