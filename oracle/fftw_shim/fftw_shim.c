/*
 * FFTW3-API subset (fftw3.h) over this repository's own CPU FFT: test infrastructure for the
 * host-core baseline, which runs the reference's lib/wderiv/c/wderiv.c unmodified.
 *
 * The transforms: per axis, powers of two by an iterative radix-2 decimation-in-time FFT
 * (bit-reversed load, log2 n butterfly passes), other lengths by a recursive mixed-radix
 * decimation in time (radices 4, 2, 3, then a direct DFT for the remaining factor).  Twiddles
 * e^{-2 pi i j / n} are tabulated per plan in long double.  A plan owns its buffers, so plans
 * are independent of each other (the baseline creates and runs them on several host threads).
 */
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include "fftw3.h"

typedef struct { double re, im; } cpx;

struct axis {
    int n;
    int pow2;
    cpx *w;        /* e^{-2 pi i j / n}, j < n */
    int *rev;      /* bit reversal of j (powers of two) */
};

struct wtd_fftw_plan_s {
    int kind;      /* 0 complex, 1 real to complex, 2 complex to real */
    int rank, n[3], sign;
    size_t total;
    void *in, *out;
    struct axis ax[3];
    cpx *work;     /* full complex field (r2c, c2r) */
    cpx *line, *scratch;
};

static cpx cmul(cpx a, cpx b) { cpx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; return r; }
static cpx cconj(cpx a) { cpx r = {a.re, -a.im}; return r; }

static int axis_init(struct axis *a, int n)
{
    a->n = n;
    a->pow2 = n > 0 && (n & (n - 1)) == 0;
    a->w = (cpx *)malloc(sizeof(cpx) * (size_t)n);
    a->rev = NULL;
    if (!a->w) return -1;
    for (int j = 0; j < n; j++) {
        const long double t = 2.0L * 3.14159265358979323846264338327950288L * (long double)j / (long double)n;
        a->w[j].re = (double)cosl(t);
        a->w[j].im = -(double)sinl(t);
    }
    if (a->pow2) {
        a->rev = (int *)malloc(sizeof(int) * (size_t)n);
        if (!a->rev) return -1;
        int bits = 0;
        while ((1 << bits) < n) bits++;
        for (int j = 0; j < n; j++) {
            int r = 0;
            for (int b = 0; b < bits; b++) r |= ((j >> b) & 1) << (bits - 1 - b);
            a->rev[j] = r;
        }
    }
    return 0;
}

/* iterative radix-2 DIT, in place, sign -1 or +1 */
static void fft_pow2(cpx *x, const struct axis *a, int sign, cpx *tmp)
{
    const int n = a->n;
    for (int j = 0; j < n; j++) tmp[a->rev[j]] = x[j];
    for (int len = 2; len <= n; len <<= 1) {
        const int half = len >> 1, step = n / len;
        for (int s = 0; s < n; s += len) {
            for (int k = 0; k < half; k++) {
                cpx w = a->w[k * step];
                if (sign > 0) w = cconj(w);
                const cpx u = tmp[s + k], v = cmul(tmp[s + k + half], w);
                tmp[s + k].re = u.re + v.re; tmp[s + k].im = u.im + v.im;
                tmp[s + k + half].re = u.re - v.re; tmp[s + k + half].im = u.im - v.im;
            }
        }
    }
    memcpy(x, tmp, sizeof(cpx) * (size_t)n);
}

/* recursive mixed-radix DIT: out[k] = sum_q in[q * stride] w^(q k), m-point sub-transforms of
 * the r decimated sequences, then r-point butterflies with twiddles */
static void fft_rec(const cpx *in, cpx *out, int n, int stride, const cpx *w, int wstep, int N, int sign, cpx *tmp)
{
    if (n == 1) { out[0] = in[0]; return; }
    const int r = (n % 4 == 0) ? 4 : (n % 2 == 0) ? 2 : (n % 3 == 0) ? 3 : n;
    const int m = n / r;
#define TW(e) (sign < 0 ? w[((long)(e) % N)] : cconj(w[((long)(e) % N)]))
    if (r == n) {
        for (int k = 0; k < n; k++) {
            cpx s = {0.0, 0.0};
            for (int q = 0; q < n; q++) {
                const cpx t = cmul(in[q * stride], TW((long)q * k % n * wstep));
                s.re += t.re; s.im += t.im;
            }
            out[k] = s;
        }
        return;
    }
    for (int q = 0; q < r; q++) fft_rec(in + q * stride, out + q * m, m, stride * r, w, wstep * r, N, sign, tmp + n);
    for (int k = 0; k < m; k++) {
        cpx t[4];
        for (int q = 0; q < r; q++) t[q] = cmul(out[q * m + k], TW((long)q * k * wstep));
        for (int j = 0; j < r; j++) {
            cpx s = {0.0, 0.0};
            for (int q = 0; q < r; q++) {
                const cpx u = cmul(t[q], TW((long)q * j * m % n * wstep));
                s.re += u.re; s.im += u.im;
            }
            tmp[k + j * m] = s;
        }
    }
    memcpy(out, tmp, sizeof(cpx) * (size_t)n);
#undef TW
}

static void transform_line(cpx *x, const struct axis *a, int sign, cpx *line, cpx *scratch)
{
    if (a->n <= 1) return;
    if (a->pow2) {
        fft_pow2(x, a, sign, scratch);
    } else {
        fft_rec(x, line, a->n, 1, a->w, 1, a->n, sign, scratch);
        memcpy(x, line, sizeof(cpx) * (size_t)a->n);
    }
}

/* unnormalised transform of a row-major complex field along every axis */
static void transform_field(cpx *f, struct wtd_fftw_plan_s *p, int sign)
{
    for (int d = 0; d < p->rank; d++) {
        const int n = p->n[d];
        size_t inner = 1, outer = 1;
        for (int b = d + 1; b < p->rank; b++) inner *= (size_t)p->n[b];
        for (int b = 0; b < d; b++) outer *= (size_t)p->n[b];
        cpx *g = p->line + n;   /* gathered line */
        for (size_t o = 0; o < outer; o++)
            for (size_t i = 0; i < inner; i++) {
                cpx *base = f + o * (size_t)n * inner + i;
                for (int j = 0; j < n; j++) g[j] = base[(size_t)j * inner];
                transform_line(g, &p->ax[d], sign, p->line, p->scratch);
                for (int j = 0; j < n; j++) base[(size_t)j * inner] = g[j];
            }
    }
}

static fftw_plan plan_new(int kind, int rank, const int *n, void *in, void *out, int sign)
{
    struct wtd_fftw_plan_s *p = (struct wtd_fftw_plan_s *)calloc(1, sizeof(*p));
    if (!p) return NULL;
    p->kind = kind; p->rank = rank; p->sign = sign; p->in = in; p->out = out;
    p->total = 1;
    int nmax = 1;
    for (int d = 0; d < rank; d++) {
        p->n[d] = n[d];
        p->total *= (size_t)n[d];
        if (n[d] > nmax) nmax = n[d];
        if (axis_init(&p->ax[d], n[d])) { fftw_destroy_plan(p); return NULL; }
    }
    /* line: result + gathered line; scratch: recursion levels of the mixed-radix transform */
    p->line = (cpx *)malloc(sizeof(cpx) * 2 * (size_t)nmax);
    p->scratch = (cpx *)malloc(sizeof(cpx) * 4 * (size_t)nmax);
    if (kind) p->work = (cpx *)malloc(sizeof(cpx) * p->total);
    if (!p->line || !p->scratch || (kind && !p->work)) { fftw_destroy_plan(p); return NULL; }
    return p;
}

fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags)
{ (void)flags; int d[1] = {n}; return plan_new(0, 1, d, in, out, sign); }
fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign, unsigned flags)
{ (void)flags; int d[2] = {n0, n1}; return plan_new(0, 2, d, in, out, sign); }
fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in, fftw_complex *out, int sign, unsigned flags)
{ (void)flags; int d[3] = {n0, n1, n2}; return plan_new(0, 3, d, in, out, sign); }
fftw_plan fftw_plan_dft_r2c_1d(int n, double *in, fftw_complex *out, unsigned flags)
{ (void)flags; int d[1] = {n}; return plan_new(1, 1, d, in, out, FFTW_FORWARD); }
fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double *in, fftw_complex *out, unsigned flags)
{ (void)flags; int d[2] = {n0, n1}; return plan_new(1, 2, d, in, out, FFTW_FORWARD); }
fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in, fftw_complex *out, unsigned flags)
{ (void)flags; int d[3] = {n0, n1, n2}; return plan_new(1, 3, d, in, out, FFTW_FORWARD); }
fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex *in, double *out, unsigned flags)
{ (void)flags; int d[1] = {n}; return plan_new(2, 1, d, in, out, FFTW_BACKWARD); }
fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex *in, double *out, unsigned flags)
{ (void)flags; int d[2] = {n0, n1}; return plan_new(2, 2, d, in, out, FFTW_BACKWARD); }
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in, double *out, unsigned flags)
{ (void)flags; int d[3] = {n0, n1, n2}; return plan_new(2, 3, d, in, out, FFTW_BACKWARD); }

/* index of the half-spectrum entry (rows of n_last/2 + 1) of full multi-index c */
static size_t half_index(const struct wtd_fftw_plan_s *p, const int *c)
{
    size_t h = 0;
    for (int d = 0; d < p->rank; d++) {
        const size_t nd = (d == p->rank - 1) ? (size_t)(p->n[d] / 2 + 1) : (size_t)p->n[d];
        h = h * nd + (size_t)c[d];
    }
    return h;
}

void fftw_execute(const fftw_plan p)
{
    if (!p) return;
    if (p->kind == 0) {
        cpx *out = (cpx *)p->out;
        if (p->out != p->in) memcpy(out, p->in, sizeof(cpx) * p->total);
        transform_field(out, p, p->sign);
        return;
    }
    const int last = p->rank - 1, nl = p->n[last];
    int c[3] = {0, 0, 0};
    if (p->kind == 1) {
        const double *in = (const double *)p->in;
        for (size_t i = 0; i < p->total; i++) { p->work[i].re = in[i]; p->work[i].im = 0.0; }
        transform_field(p->work, p, FFTW_FORWARD);
        cpx *out = (cpx *)p->out;
        for (size_t i = 0; i < p->total; i++) {
            size_t r = i;
            for (int d = last; d >= 0; d--) { c[d] = (int)(r % (size_t)p->n[d]); r /= (size_t)p->n[d]; }
            if (c[last] <= nl / 2) out[half_index(p, c)] = p->work[i];
        }
        return;
    }
    /* complex to real: the full spectrum from the half one, X(-k) = conj X(k) */
    const cpx *in = (const cpx *)p->in;
    for (size_t i = 0; i < p->total; i++) {
        size_t r = i;
        for (int d = last; d >= 0; d--) { c[d] = (int)(r % (size_t)p->n[d]); r /= (size_t)p->n[d]; }
        if (c[last] <= nl / 2) {
            p->work[i] = in[half_index(p, c)];
        } else {
            int m[3];
            for (int d = 0; d <= last; d++) m[d] = (p->n[d] - c[d]) % p->n[d];
            p->work[i] = cconj(in[half_index(p, m)]);
        }
    }
    transform_field(p->work, p, FFTW_BACKWARD);
    double *out = (double *)p->out;
    for (size_t i = 0; i < p->total; i++) out[i] = p->work[i].re;
}

void fftw_destroy_plan(fftw_plan p)
{
    if (!p) return;
    for (int d = 0; d < 3; d++) { free(p->ax[d].w); free(p->ax[d].rev); }
    free(p->work); free(p->line); free(p->scratch);
    free(p);
}
