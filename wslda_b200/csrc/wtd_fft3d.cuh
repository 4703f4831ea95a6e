/*
 * Spectral derivatives of fields too large for one CTA's shared memory (3D 32^3, 48^3 ...; 2D
 * beyond about 74x74 in FP64): a plane/pencil decomposition through global memory.  In 2D a
 * "plane" is one contiguous row along y.
 *
 *   k_planes  : one CTA per (field, x-plane) — 2D FFT over (y, z) of a contiguous plane in smem
 *   k_pencils : one CTA per (field, group of PX consecutive (y, z) pencils) — FFT along x,
 *               then for every requested operator: multiply by -|k|^2/N or i k_d/N (Nyquist
 *               zeroed for first derivatives, pca_derivative.cu:152-171), inverse FFT along x,
 *               store.  The (y, z) wave numbers come from the digit-reversed plane positions.
 *   inverse planes on every output.
 *
 * A derivative set of nf fields costs 1 + nops + 2*nops array passes of reads and writes
 * (laplacian only: 3 reads + 3 writes), against the reference's cuFFT forward, multiply
 * kernel and one cuFFT inverse per output (pca_derivative.cu:217-277).
 */
#ifndef WTD_FFT3D_CUH
#define WTD_FFT3D_CUH

#include "wtd_step.cuh"

/* pencils per CTA: 16, or the largest power of two dividing NY*NZ (even, as every lattice
 * extent the reference accepts) */
#define WTD_NYZ ((NY) * (NZ))
#define WTD_PX (WTD_NYZ % 16 == 0 ? 16 : WTD_NYZ % 8 == 0 ? 8 : WTD_NYZ % 4 == 0 ? 4 : 2)

/* 2D (y, z) transform of plane x of field f: in -> out (may alias), fields of N points each */
template <class GP, int SIGN>
__global__ void __launch_bounds__(512) k_planes(const double2 *in, double2 *out, int nx, const double2 *gtw_yz, const double *gk)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *B = (double2 *)smem_raw;
    double2 *tw = B + GP::padded;
    double (*kt)[WTD_KT] = (double (*)[WTD_KT])(tw + GP::twtotal);
    (void)kt;
    (void)nx;
    for (int t = threadIdx.x; t < GP::N0 + GP::N1; t += blockDim.x) tw[t] = gtw_yz[t];
    constexpr int NP = GP::ntot;
    const size_t base = (size_t)blockIdx.x * NP;   /* blockIdx.x = f * nx + x: planes are contiguous */
    for (int p = threadIdx.x; p < NP; p += blockDim.x) B[GP::off(p)] = in[base + p];
    __syncthreads();
    if (SIGN < 0) fft_forward<GP, 1>(B, 0, tw);
    else fft_inverse<GP, 1>(B, 0, tw);
    for (int p = threadIdx.x; p < NP; p += blockDim.x) out[base + p] = B[GP::off(p)];
}

/* x-pencil pass: forward x FFT, then per operator multiply + inverse x FFT.
 * in: fields already (y, z)-transformed; out[op] gets op applied (still (y, z)-transformed).
 * ops bit 0: laplacian, bit 1..3: d/dx, d/dy, d/dz.  Outputs may alias the input. */
template <class GX>
__global__ void __launch_bounds__(512) k_pencils(const double2 *in, double2 *olap, double2 *odx, double2 *ody, double2 *odz,
                                                 int nyz, int N, const double2 *gtw_x, const double *gk,
                                                 int filt, double fmu, double fT)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *B0 = (double2 *)smem_raw;
    double2 *W = B0 + GX::padded;
    double2 *tw = W + GX::padded;
    double (*kt)[WTD_KT] = (double (*)[WTD_KT])(tw + GX::twtotal);
    constexpr int NXL = GX::N0, PX = GX::N1;
    for (int t = threadIdx.x; t < NXL; t += blockDim.x) tw[t] = gtw_x[t];
    for (int t = threadIdx.x; t < 6 * WTD_KT; t += blockDim.x) kt[t / WTD_KT][t % WTD_KT] = gk[t];
    const int groups = nyz / PX;
    const int f = blockIdx.x / groups, g = blockIdx.x - f * groups;
    const size_t fb = (size_t)f * N;
    const int q0 = g * PX;
    /* element (x, q) of the field sits at x*nyz + q */
    for (int i = threadIdx.x; i < NXL * PX; i += blockDim.x) {
        int x = i / PX, j = i - x * PX;
        B0[GX::off(x * PX + j)] = in[fb + (size_t)x * nyz + q0 + j];
    }
    __syncthreads();
    fft_axis_fwd<GX, 0, 0, NXL, 1>(B0, 0, tw);
    double2 *outs[4] = {olap, odx, ody, odz};
    for (int op = 0; op < 4; op++) {
        double2 *o = outs[op];
        if (!o) continue;
        for (int i = threadIdx.x; i < NXL * PX; i += blockDim.x) {
            int x = i / PX, j = i - x * PX;
            int q = q0 + j;
            int yq = q / NZ, zq = q - yq * NZ;
            double2 z = B0[GX::off(x * PX + j)];
            double2 r;
            if (op == 0) {
                /* laplacian -|k|^2/N, or (filt) the high-k filter FD(|k|^2/2)/N into olap */
                double kx = kt[0][x], ky = kt[1][yq], kz = kt[2][zq];
                double k2 = kx * kx + ky * ky + kz * kz;
                double s = filt ? 1.0 / (exp((0.5 * k2 - fmu) / fT) + 1.0) / (double)N : -1.0 * k2 / (double)N;
                r = make_double2(z.x * s, z.y * s);
            } else {
                double k = (op == 1) ? kt[3][x] : (op == 2) ? kt[4][yq] : kt[5][zq];
                double s = k / (double)N;
                r = make_double2(-s * z.y, s * z.x);
            }
            W[GX::off(x * PX + j)] = r;
        }
        __syncthreads();
        fft_axis_inv<GX, 0, NXL, 1>(W, 0, tw);
        for (int i = threadIdx.x; i < NXL * PX; i += blockDim.x) {
            int x = i / PX, j = i - x * PX;
            o[fb + (size_t)x * nyz + q0 + j] = W[GX::off(x * PX + j)];
        }
        __syncthreads();
    }
}

typedef Geo<NY, NZ, 1> WGP;          /* one (y, z) plane */
typedef Geo<NX, WTD_PX, 1> WGX;      /* PX pencils along x */

static constexpr size_t planes_smem = (size_t)WGP::padded * sizeof(double2) + WGP::twtotal * sizeof(double2) + sizeof(KTab<WGP>);
static constexpr size_t pencils_smem = 2 * (size_t)WGX::padded * sizeof(double2) + WGX::twtotal * sizeof(double2) + sizeof(KTab<WGX>);

/* twiddles of the plane geometry start at the y axis of the lattice table (offset NX) and of
 * the pencil geometry at the x axis (offset 0): both are e^{-2 pi i t/n} per axis */
static int big_derivs(double2 *in, int nf, double2 *lap, double2 *dx, double2 *dy, double2 *dz,
                      const double2 *tw, const double *ktab, cudaStream_t st, int filt = 0, double fmu = 0.0,
                      double fT = 1.0)
{
    constexpr int NYZ = NY * NZ, N = NX * NY * NZ;
    if (NYZ % WTD_PX != 0) return WTD_ERR_UNSUPPORTED;
    WTD_ONCE_PER_DEVICE(
        WTD_CU(cudaFuncSetAttribute(k_planes<WGP, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)planes_smem));
        WTD_CU(cudaFuncSetAttribute(k_planes<WGP, +1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)planes_smem));
        WTD_CU(cudaFuncSetAttribute(k_pencils<WGX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pencils_smem)));
    /* forward (y, z) into the laplacian buffer (in place when there is none: the input is then
     * overwritten by its transform) */
    double2 *K = lap ? lap : in;
    k_planes<WGP, -1><<<nf * NX, 512, planes_smem, st>>>(in, K, NX, tw + NX, ktab);
    k_pencils<WGX><<<nf * (NYZ / WTD_PX), 512, pencils_smem, st>>>(K, lap, dx, dy, dz, NYZ, N, tw, ktab, filt, fmu, fT);
    double2 *outs[4] = {lap, dx, dy, dz};
    for (int k = 0; k < 4; k++)
        if (outs[k]) k_planes<WGP, +1><<<nf * NX, 512, planes_smem, st>>>(outs[k], outs[k], NX, tw + NX, ktab);
    return cudaGetLastError() == cudaSuccess ? WTD_OK : WTD_ERR_CUDA;
}

/* ---------------------------------------------------------------------------------------
 * Separable derivative sets of the state fields.  The multipliers of d/dy, d/dz and of the
 * (y, z) part of the laplacian do not depend on k_x, and those of d/dx and of the x part do not
 * depend on (k_y, k_z).  The transforms along the other axes therefore cancel:
 *
 *   d/dy f = IFFT_yz[i k_y FFT_yz f] / (NY NZ)          d/dx f = IFFT_x[i k_x FFT_x f] / NX
 *   lap f  = IFFT_yz[-(k_y^2 + k_z^2) FFT_yz f] / (NY NZ) + IFFT_x[-k_x^2 FFT_x f] / NX
 *
 * with the reference's Nyquist zeroing of first derivatives (pca_derivative.cu:152-171).  Two
 * passes, no transpose between CTAs:
 *   k_sep_planes : one CTA per (field, x plane): d/dy, d/dz and the (y, z) part of lap;
 *   k_sep_pencils: one CTA per (field, group of x pencils): d/dx, and lap += its x part.
 * A full set costs 3 reads + 5 writes of the fields, a laplacian 3 reads + 2 writes, against
 * 6 + 9 and 3 + 3 for big_derivs.  Optional point weights multiply field f by wa (f < nfa) or
 * wb before the transforms: lap(alpha psi) of the variable-mass kinetic term
 * (multiply_wf_by_alpha + compute_laplace, pca.c:1455-1456) in one go.
 * The input must not alias an output.
 * -------------------------------------------------------------------------------------*/
#define WTD_SEP_NT 256
/* pencils per CTA of the x pass: up to 32 (512-byte rows), at most 2048 points, dividing NY*NZ */
#define WTD_PXS_CAP (2048 / (NX) >= 32 ? 32 : 2048 / (NX) >= 16 ? 16 : 2048 / (NX) >= 8 ? 8 : 4)
#define WTD_PXS (WTD_NYZ % WTD_PXS_CAP == 0 ? WTD_PXS_CAP : WTD_PX)

/* CTAs per SM asked of the register allocator for the plane kernel: 4 (at most 64 registers a
 * thread; the plane FFT stages are latency-bound, and the register file otherwise admits 3)
 * where 4 CTAs' shared memory fits an SM (228 KB, 1 KB reserved per CTA), else as many as fit */
template <class GP> struct SepPlanesMinB {
    static constexpr size_t smem = 2 * (size_t)GP::padded * sizeof(double2) + GP::twtotal * sizeof(double2) + sizeof(KTab<GP>);
    static constexpr size_t per = smem + 1024, sm = 233472;
    static constexpr int value = 4 * per <= sm ? 4 : 3 * per <= sm ? 3 : 2 * per <= sm ? 2 : 1;
};
template <class GP>
__global__ void __launch_bounds__(WTD_SEP_NT, SepPlanesMinB<GP>::value) k_sep_planes(const double2 *__restrict__ in, double2 *lap, double2 *dy,
                                                          double2 *dz, const double *wa, const double *wb, int nfa,
                                                          const double2 *gtw_yz, const double *gk)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *B = (double2 *)smem_raw;
    double2 *W = B + GP::padded;
    double2 *tw = W + GP::padded;
    double (*kt)[WTD_KT] = (double (*)[WTD_KT])(tw + GP::twtotal);
    constexpr int NP = GP::ntot;
    for (int t = threadIdx.x; t < GP::N0 + GP::N1; t += WTD_SEP_NT) tw[t] = gtw_yz[t];
    for (int t = threadIdx.x; t < 6 * WTD_KT; t += WTD_SEP_NT) kt[t / WTD_KT][t % WTD_KT] = gk[t];
    const int f = blockIdx.x / NX, x = blockIdx.x - f * NX;
    const size_t base = (size_t)blockIdx.x * NP;   /* planes of a field are contiguous */
    const double *w = wa ? (f < nfa ? wa : wb) + (size_t)x * NP : nullptr;
    for (int p = threadIdx.x; p < NP; p += WTD_SEP_NT) {
        double2 z = in[base + p];
        if (w) {
            const double a = w[p];
            z = make_double2(z.x * a, z.y * a);
        }
        B[GP::off(p)] = z;
    }
    __syncthreads();
    fft_forward<GP, 1>(B, 0, tw);
    const double inv = 1.0 / (double)NP;
#pragma unroll
    for (int op = 0; op < 3; op++) {
        double2 *o = op == 0 ? dy : op == 1 ? dz : lap;
        if (!o) continue;
        double2 *T = (op == 2) ? B : W; /* the laplacian comes last and works in place */
        for (int p = threadIdx.x; p < NP; p += WTD_SEP_NT) {
            const int yq = p / NZ, zq = p - yq * NZ;
            const double2 z = B[GP::off(p)];
            double2 r;
            if (op == 2) {
                const double ky = kt[1][yq], kz = kt[2][zq];
                const double sc = -(ky * ky + kz * kz) * inv;
                r = make_double2(z.x * sc, z.y * sc);
            } else {
                const double k = (op == 0 ? kt[4][yq] : kt[5][zq]) * inv;
                r = make_double2(-k * z.y, k * z.x);
            }
            T[GP::off(p)] = r;
        }
        __syncthreads();
        fft_inverse<GP, 1>(T, 0, tw);
        for (int p = threadIdx.x; p < NP; p += WTD_SEP_NT) o[base + p] = T[GP::off(p)];
        __syncthreads();
    }
}

template <class GX>
__global__ void __launch_bounds__(WTD_SEP_NT) k_sep_pencils(const double2 *__restrict__ in, double2 *lap, double2 *dx,
                                                           const double *wa, const double *wb, int nfa,
                                                           const double2 *gtw_x, const double *gk)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *B = (double2 *)smem_raw;
    double2 *W = B + GX::padded;
    double2 *tw = W + GX::padded;
    double (*kt)[WTD_KT] = (double (*)[WTD_KT])(tw + GX::twtotal);
    constexpr int NXL = GX::N0, PX = GX::N1, NYZ = NY * NZ, N = NX * NY * NZ, groups = NYZ / PX;
    for (int t = threadIdx.x; t < NXL; t += WTD_SEP_NT) tw[t] = gtw_x[t];
    for (int t = threadIdx.x; t < 6 * WTD_KT; t += WTD_SEP_NT) kt[t / WTD_KT][t % WTD_KT] = gk[t];
    const int f = blockIdx.x / groups, g = blockIdx.x - f * groups;
    const size_t fb = (size_t)f * N;
    const int q0 = g * PX;
    const double *w = wa ? (f < nfa ? wa : wb) : nullptr;
    /* element (x, q) of the field sits at x*NYZ + q */
    for (int i = threadIdx.x; i < NXL * PX; i += WTD_SEP_NT) {
        const int x = i / PX, j = i - x * PX;
        const size_t pt = (size_t)x * NYZ + q0 + j;
        double2 z = in[fb + pt];
        if (w) {
            const double a = w[pt];
            z = make_double2(z.x * a, z.y * a);
        }
        B[GX::off(i)] = z;
    }
    __syncthreads();
    fft_axis_fwd<GX, 0, 0, NXL, 1>(B, 0, tw);
    const double inv = 1.0 / (double)NXL;
    if (dx) {
        for (int i = threadIdx.x; i < NXL * PX; i += WTD_SEP_NT) {
            const int x = i / PX;
            const double k = kt[3][x] * inv;
            const double2 z = B[GX::off(i)];
            W[GX::off(i)] = make_double2(-k * z.y, k * z.x);
        }
        __syncthreads();
        fft_axis_inv<GX, 0, NXL, 1>(W, 0, tw);
        for (int i = threadIdx.x; i < NXL * PX; i += WTD_SEP_NT) {
            const int x = i / PX, j = i - x * PX;
            dx[fb + (size_t)x * NYZ + q0 + j] = W[GX::off(i)];
        }
    }
    if (lap) {
        /* each thread scales the elements it reads: no barrier needed before the in-place write */
        for (int i = threadIdx.x; i < NXL * PX; i += WTD_SEP_NT) {
            const int x = i / PX;
            const double kx = kt[0][x];
            const double sc = -(kx * kx) * inv;
            const double2 z = B[GX::off(i)];
            B[GX::off(i)] = make_double2(z.x * sc, z.y * sc);
        }
        __syncthreads();
        fft_axis_inv<GX, 0, NXL, 1>(B, 0, tw);
        for (int i = threadIdx.x; i < NXL * PX; i += WTD_SEP_NT) {
            const int x = i / PX, j = i - x * PX;
            const size_t a = fb + (size_t)x * NYZ + q0 + j;
            const double2 yz = lap[a], xp = B[GX::off(i)];
            lap[a] = make_double2(yz.x + xp.x, yz.y + xp.y);
        }
    }
}

typedef Geo<NX, WTD_PXS, 1> WGXS;    /* WTD_PXS pencils along x */
static constexpr size_t sep_planes_smem = 2 * (size_t)WGP::padded * sizeof(double2) + WGP::twtotal * sizeof(double2) + sizeof(KTab<WGP>);
static constexpr size_t sep_pencils_smem = 2 * (size_t)WGXS::padded * sizeof(double2) + WGXS::twtotal * sizeof(double2) + sizeof(KTab<WGXS>);

/* lap, d/dx, d/dy, d/dz (any may be NULL) of nf fields of N points; wa/wb: optional weights */
static int big_derivs_sep(const double2 *in, int nf, double2 *lap, double2 *dx, double2 *dy, double2 *dz,
                          const double *wa, const double *wb, const double2 *tw, const double *ktab, cudaStream_t st)
{
    constexpr int NYZ = NY * NZ;
    if (NYZ % WTD_PXS != 0) return WTD_ERR_UNSUPPORTED;
    if (sep_planes_smem > WTD_SMEM_MAX || sep_pencils_smem > WTD_SMEM_MAX) return WTD_ERR_UNSUPPORTED;
    if (in == lap || in == dx || in == dy || in == dz) return WTD_ERR_ARG;
    WTD_ONCE_PER_DEVICE(
        WTD_CU(cudaFuncSetAttribute(k_sep_planes<WGP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sep_planes_smem));
        WTD_CU(cudaFuncSetAttribute(k_sep_planes<WGP>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                    (int)cudaSharedmemCarveoutMaxShared));
        WTD_CU(cudaFuncSetAttribute(k_sep_pencils<WGXS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sep_pencils_smem)));
    const int nfa = nf / 2;
    if (lap || dy || dz)
        k_sep_planes<WGP><<<nf * NX, WTD_SEP_NT, sep_planes_smem, st>>>(in, lap, dy, dz, wa, wb, nfa, tw + NX, ktab);
    if (lap || dx)
        k_sep_pencils<WGXS><<<nf * (NYZ / WTD_PXS), WTD_SEP_NT, sep_pencils_smem, st>>>(in, lap, dx, wa, wb, nfa, tw, ktab);
    return cudaGetLastError() == cudaSuccess ? WTD_OK : WTD_ERR_CUDA;
}

/* real field -> laplacian or d/dx_d of it (complex staging buffer of N points) */
__global__ void k_real_to_c(const double *f, double2 *c, int n)
{
    int i = threadIdx.x + blockIdx.x * blockDim.x;
    if (i < n) c[i] = make_double2(f[i], 0.0);
}
__global__ void k_c_to_real(const double2 *c, double *f, int n, double scale, int accumulate)
{
    int i = threadIdx.x + blockIdx.x * blockDim.x;
    if (i < n) f[i] = accumulate ? f[i] + scale * c[i].x : scale * c[i].x;
}
/* tau = max(0, lap(rho)/2 - tau_tmp) from the staged laplacian (pca_dens.cu:275-290) */
__global__ void k_tau_from_lap(const double2 *lap, double *tau, int n)
{
    int i = threadIdx.x + blockIdx.x * blockDim.x;
    if (i >= n) return;
    double t = 0.5 * lap[i].x - tau[i];
    tau[i] = t < 0.0 ? 0.0 : t;
}

/* out (+)= scale * op(f) for a real field: which 0 = laplacian, 1..3 = d/dx, d/dy, d/dz.
 * stage holds 2N complex numbers of scratch. */
static int big_real_deriv(const double *f, double *out, int which, double scale, int accumulate, double2 *stage,
                          const double2 *tw, const double *kt, cudaStream_t st)
{
    constexpr int N = NX * NY * NZ;
    const int nb = (N + 255) / 256;
    k_real_to_c<<<nb, 256, 0, st>>>(f, stage, N);
    double2 *res = stage;
    int r;
    if (which == 0) r = big_derivs(stage, 1, stage, NULL, NULL, NULL, tw, kt, st);
    else {
        res = stage + N;
        r = big_derivs(stage, 1, NULL, which == 1 ? res : NULL, which == 2 ? res : NULL, which == 3 ? res : NULL, tw, kt, st);
    }
    if (r) return r;
    k_c_to_real<<<nb, 256, 0, st>>>(res, out, N, scale, accumulate);
    return cudaGetLastError() == cudaSuccess ? WTD_OK : WTD_ERR_CUDA;
}

/* high-k filter of nf consecutive real fields of N doubles, in place (large lattices);
 * stage holds N complex numbers of scratch */
static int big_filter_real(double *f, int nf, double mu, double T, double2 *stage, const double2 *tw, const double *kt,
                           cudaStream_t st)
{
    constexpr int N = NX * NY * NZ;
    const int nb = (N + 255) / 256;
    for (int k = 0; k < nf; k++) {
        k_real_to_c<<<nb, 256, 0, st>>>(f + (size_t)k * N, stage, N);
        WTD_TRY(big_derivs(stage, 1, stage, NULL, NULL, NULL, tw, kt, st, 1, mu, T));
        k_c_to_real<<<nb, 256, 0, st>>>(stage, f + (size_t)k * N, N, 1.0, 0);
    }
    return cudaGetLastError() == cudaSuccess ? WTD_OK : WTD_ERR_CUDA;
}

/* tau of both spins on a large lattice */
static int big_tau(double *dens, double2 *stage, const double2 *tw, const double *kt, cudaStream_t st)
{
    constexpr int N = NX * NY * NZ;
    const int nb = (N + 255) / 256;
    for (int s = 0; s < 2; s++) {
        k_real_to_c<<<nb, 256, 0, st>>>(dens + (s == 0 ? 2 : 7) * (size_t)N, stage, N);
        int r = big_derivs(stage, 1, stage, NULL, NULL, NULL, tw, kt, st);
        if (r) return r;
        k_tau_from_lap<<<nb, 256, 0, st>>>(stage, dens + (s == 0 ? 3 : 8) * (size_t)N, N);
    }
    return cudaGetLastError() == cudaSuccess ? WTD_OK : WTD_ERR_CUDA;
}

/* variable mass on a large lattice: CF_NA/NB = lap(alpha)/4, CF_CJA/CJB = -div(A)/2
 * (pca_kernels.cu:778-795), from the CF_ALA.. / CF_AAX.. rows already in cf */
static int big_prep_var(double *cf, double2 *stage, const double2 *tw, const double *kt, cudaStream_t st)
{
    constexpr size_t N = (size_t)NX * NY * NZ;
    for (int s = 0; s < 2; s++) {
        WTD_TRY(big_real_deriv(cf + (s == 0 ? CF_ALA : CF_ALB) * N, cf + (s == 0 ? CF_NA : CF_NB) * N, 0, 0.25, 0, stage, tw, kt, st));
        for (int d = 0; d < 3; d++)
            WTD_TRY(big_real_deriv(cf + ((s == 0 ? CF_AAX : CF_ABX) + d) * N, cf + (s == 0 ? CF_CJA : CF_CJB) * N, d + 1, -0.5,
                                   d > 0, stage, tw, kt, st));
    }
    return WTD_OK;
}

#endif
