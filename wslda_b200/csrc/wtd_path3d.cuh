/*
 * The line path: one TD half step on 3D lattices whose state does not fit one CTA (32^3,
 * 48^3, ...), as three kernels per half step instead of the reference's ~30 whole-array
 * kernels (hpc-engine/pca.c:1401-1571):
 *
 *   k3_plane_h    one CTA per (field, x-plane): the (y, z) part of the kinetic and current
 *                 terms of H psi, K_yz, by 1D spectral derivatives along the y- and z-lines of
 *                 the plane (pca_derivative.cu:217-277, pca_kernels.cu:233-391, 981-1026):
 *                     K_yz = s a (lap_y + lap_z) psi + (-i A_y) d_y psi + (-i A_z) d_z psi
 *                            - s/4 (lap_y + lap_z)(alpha psi)         (variable mass)
 *                     K_yz = s a (lap_y + lap_z) psi                   (constant mass)
 *                 with s = +1 for u, -1 for v and a the CF_AA/CF_AB coefficient.
 *   k3_xline      a thread-block cluster per state, each CTA a slab of (y, z) columns, one
 *                 thread per (component, column): the x-line part of H psi added to K_yz and
 *                 the local terms, <H> (cluster sum through distributed shared memory), the
 *                 ABM predictor or corrector (tdwslda_ode_integrator.h:26-220), the norm
 *                 (cluster sum), renormalisation and store, the rho and nu partial sums and,
 *                 on gradient half steps, the x-parts of tau and j (pca_dens.cu:13-198).
 *   k3_plane_dens on gradient half steps, one CTA per (component, x-plane, chunk of states):
 *                 the y- and z-parts of tau and j of the updated states, summed over the
 *                 chunk in shared memory, one slot write per CTA.
 *
 * Every transform is a register-resident line FFT (wtd_line.cuh); the separable multipliers
 * (d/dx_d and lap = sum_d d^2/dx_d^2 act along one axis each) make three 1D transforms per
 * derivative set instead of a 3D one, with 1/n_d folded into the multipliers.  HBM traffic per
 * half step is the compulsory ABM stream plus one read and one write of K_yz and one read of
 * the updated state for the gradient part.
 *
 * Precision forms as in the fused 2D pass: TY storage of the states, TH of the ABM history,
 * TC of the transforms and H psi; the ABM sums, norms, <H> and density sums are FP64.
 */
#ifndef WTD_PATH3D_CUH
#define WTD_PATH3D_CUH

#include <cooperative_groups.h>
#include "wtd_line.cuh"

#if CODEDIM == 3
#define WTD_L_NMAX ((NX) > (NY) ? ((NX) > (NZ) ? (NX) : (NZ)) : ((NY) > (NZ) ? (NY) : (NZ)))
#define WTD_L_NYZ ((NY) * (NZ))

/* threads sharing one line of n points: 4 where 16 divides n, else 2 where 4 divides n, else 1 */
__host__ __device__ constexpr int line_team(int n) { return n % 16 == 0 ? 4 : n % 4 == 0 ? 2 : 1; }

/* the (comp, point) coefficient of the CF_* list */
#define CFP(k, p) cf[(size_t)(k) * (size_t)WTD_NUMEL + (p)]

/* geometry of the plane kernels: y-lines (one per z, NY points, TY threads each), then z-lines
 * (one per y, NZ points, TZ threads each) of one (y, z) plane per CTA */
struct PlaneGeo {
    static constexpr int TY = line_team(NY), TZ = line_team(NZ);
    static constexpr int AY = NZ * TY, AZ = NY * TZ;                /* active threads per phase */
    static constexpr int PT = ((AY > AZ ? AY : AZ) + 31) / 32 * 32;
    static constexpr int PITCH = NZ + 2;                            /* padded plane row */
    static constexpr int SCR = (NZ * team_scratch(NY, TY) > NY * team_scratch(NZ, TZ)) ? NZ * team_scratch(NY, TY)
                                                                                         : NY * team_scratch(NZ, TZ);
    /* whole warps in every phase: the team exchanges synchronise full warps */
    static constexpr bool ok = AY % 32 == 0 && AZ % 32 == 0;
};

template <typename TC> struct PlaneSmem {
    typedef typename cplx<TC>::t C;
    static constexpr size_t plane = (size_t)(NY) * PlaneGeo::PITCH * sizeof(C);
    static constexpr size_t scr = (size_t)PlaneGeo::SCR * sizeof(C);
    static constexpr size_t tab = (sizeof(LineTab<TC, WTD_L_NMAX>) + 15) / 16 * 16;
    /* k3_plane_h: table, the CTA's coefficient planes (compute precision, plane layout:
     * variable mass alpha, A_y, A_z and the kinetic coefficient of the component; constant
     * mass the kinetic coefficient), then per state in flight a psi plane, a K plane and the
     * team scratch.  Two states per CTA where that still leaves two CTAs per SM. */
    static constexpr int NCF = WTD_VAR ? 4 : 1;
    static constexpr size_t cfp = ((size_t)NCF * (NY) * PlaneGeo::PITCH * sizeof(TC) + 15) / 16 * 16;
    static constexpr size_t hstate = 2 * plane + scr;
    static constexpr int HS = (tab + cfp + 2 * hstate) * 2 + 2048 <= WTD_SMEM_MAX ? 2 : 1;
    static constexpr size_t h_bytes = tab + cfp + (size_t)HS * hstate;
    /* k3_plane_dens: table, psi plane, team scratch, three FP64 accumulators */
    static constexpr size_t d_bytes = tab + plane + scr + 3 * (size_t)WTD_L_NYZ * sizeof(double);
};

/* one axis of a plane for one team: the line's n/T points at plane positions pos(i) */
template <int n, int T, typename TC, bool VAR>
__device__ __forceinline__ void plane_h_axis(const typename cplx<TC>::t *P, typename cplx<TC>::t *Kp,
                                            typename cplx<TC>::t *scr, const LineTab<TC, WTD_L_NMAX> &Tb, int ax,
                                            int g, int line, const TC *cfs, int comp, bool first)
{
    typedef typename cplx<TC>::t C;
    constexpr int n1 = n / T, PITCH = PlaneGeo::PITCH;
    const bool yl = ax == 1;
    /* smem index and lattice index of slice point i (the line coordinate is g + T i) */
    auto at = [&](int i) -> int { const int c = g + T * i; return yl ? c * PITCH + line : line * PITCH + c; };
    constexpr int PL = (NY) * PITCH;                   /* one coefficient plane */
    const TC *lapk = Tb.lapk[ax], *dk = Tb.dk[ax];
    const C *tw = Tb.tw[ax];
    const TC sgn = comp ? (TC)-1 : (TC)1;
    C v[n1], w[n1];
    if (VAR) {
#pragma unroll
        for (int i = 0; i < n1; i++) {
            const TC al = cfs[at(i)];
            v[i] = P[at(i)];
            v[i].x *= al; v[i].y *= al;
        }
        team_fwd<n, T>(v, scr, g, tw);
        team_mul_lap<n, T>(v, lapk, g);
        team_inv<n, T>(v, scr, g, tw);
        /* the plane's K values of the line are read before any is written (here and below), so
         * that the shared-memory round trips overlap */
        C hk[n1];
#pragma unroll
        for (int i = 0; i < n1; i++) {
            if (first) { hk[i].x = (TC)0; hk[i].y = (TC)0; } else hk[i] = Kp[at(i)];
        }
#pragma unroll
        for (int i = 0; i < n1; i++) {
            C h = hk[i];
            h.x += sgn * (TC)-0.25 * v[i].x; h.y += sgn * (TC)-0.25 * v[i].y;
            Kp[at(i)] = h;
        }
    }
#pragma unroll
    for (int i = 0; i < n1; i++) v[i] = P[at(i)];
    team_fwd<n, T>(v, scr, g, tw);
    if (VAR) {
#pragma unroll
        for (int i = 0; i < n1; i++) w[i] = v[i];
        team_mul_d<n, T>(w, dk, g);
        team_inv<n, T>(w, scr, g, tw);
        C hk[n1];
#pragma unroll
        for (int i = 0; i < n1; i++) hk[i] = Kp[at(i)];
#pragma unroll
        for (int i = 0; i < n1; i++) {
            const TC A = cfs[ax * PL + at(i)];
            C h = hk[i];
            h.x += A * w[i].y; h.y += -A * w[i].x;
            Kp[at(i)] = h;
        }
    }
    team_mul_lap<n, T>(v, lapk, g);
    team_inv<n, T>(v, scr, g, tw);
    C hk[n1];
#pragma unroll
    for (int i = 0; i < n1; i++) {
        if (first && !VAR) { hk[i].x = (TC)0; hk[i].y = (TC)0; } else hk[i] = Kp[at(i)];
    }
#pragma unroll
    for (int i = 0; i < n1; i++) {
        const TC a = sgn * cfs[(VAR ? 3 : 0) * PL + at(i)];
        C h = hk[i];
        h.x += a * v[i].x; h.y += a * v[i].y;
        Kp[at(i)] = h;
    }
}

/* ---------------------------------------------------------------------------------------
 * k3_plane_h
 * -------------------------------------------------------------------------------------*/
template <typename TY, typename TC, bool VAR>
__global__ void __launch_bounds__(PlaneGeo::PT * PlaneSmem<TC>::HS) k3_plane_h(const TY *__restrict__ Y,
                                                                             typename cplx<TC>::t *__restrict__ K,
                                                                             const double *__restrict__ cf, int S,
                                                                             const double2 *gtw, const double *gk)
{
    typedef typename cplx<TC>::t C;
    typedef PlaneSmem<TC> SM;
    typedef PlaneGeo PG;
    constexpr int N = WTD_NUMEL, NYZ = WTD_L_NYZ, PT = PG::PT, PITCH = PG::PITCH, HS = SM::HS, PL = (NY) * PITCH;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    LineTab<TC, WTD_L_NMAX> &Tb = *(LineTab<TC, WTD_L_NMAX> *)smem_raw;
    TC *CFs = (TC *)(smem_raw + SM::tab);
    /* this CTA's (component, x-plane) pair, the same for every state it processes; its states
     * are chunk, chunk + nch, ... split over the HS halves of the CTA */
    const int pairs = 2 * NX, pr = (int)(blockIdx.x % pairs), chunk = (int)(blockIdx.x / pairs);
    const int nch = (int)(gridDim.x / pairs);
    const int comp = pr / NX, x = pr - comp * NX;
    const int half = threadIdx.x / PT, t = threadIdx.x - half * PT;
    C *P = (C *)(smem_raw + SM::tab + SM::cfp + (size_t)half * SM::hstate);
    C *Kp = P + PL;
    C *Sc = Kp + PL;
    line_tables<TC, WTD_L_NMAX, NX, NY, NZ>(Tb, gtw, gk, WTD_KT);
    /* the pair's coefficients, once per launch */
    for (int k = 0; k < SM::NCF; k++) {
        const int cfk = VAR ? (k == 0 ? CF_ALA + comp : k == 1 ? (comp ? CF_ABY : CF_AAY) : k == 2 ? (comp ? CF_ABZ : CF_AAZ)
                                                                                          : CF_AA + comp)
                            : CF_AA + comp;
        const double *src = cf + (size_t)cfk * N + (size_t)x * NYZ;
        for (int i = threadIdx.x; i < NYZ; i += blockDim.x) CFs[k * PL + (i / NZ) * PITCH + (i % NZ)] = (TC)src[i];
    }
    __syncthreads();
    for (int n0 = HS * chunk; n0 < S; n0 += HS * nch) {
        const int n = n0 + half;
        const bool act = n < S;                          /* uniform per half (whole warps) */
        const size_t base = ((size_t)comp * S + n) * N + (size_t)x * NYZ;   /* the plane's first point */
        const LineTab<TC, WTD_L_NMAX> &T = *opaque_ptr(&Tb);
        const TC *cfs = opaque_ptr((const TC *)CFs);
        if (t == 0 && act && n + HS * nch < S) prefetch_l2(Y + base + (size_t)HS * nch * N, (size_t)NYZ * sizeof(TY));
        if (act)
            for (int i = t; i < NYZ; i += PT) {
                const double2 a = to_d(Y[base + i]);
                C c; c.x = (TC)a.x; c.y = (TC)a.y;
                P[(i / NZ) * PITCH + (i % NZ)] = c;
            }
        __syncthreads();
        if (act && t < PG::AY) {
            const int line = t / PG::TY, g = t - line * PG::TY;
            plane_h_axis<NY, PG::TY, TC, VAR>(P, Kp, Sc + line * Team<NY, PG::TY>::scratch, T, 1, g, line, cfs, comp, true);
        }
        __syncthreads();
        if (act && t < PG::AZ) {
            const int line = t / PG::TZ, g = t - line * PG::TZ;
            plane_h_axis<NZ, PG::TZ, TC, VAR>(P, Kp, Sc + line * Team<NZ, PG::TZ>::scratch, T, 2, g, line, cfs, comp, false);
        }
        __syncthreads();
        if (act)
            for (int i = t; i < NYZ; i += PT) K[base + i] = Kp[(i / NZ) * PITCH + (i % NZ)];
        __syncthreads();
    }
}

/* ---------------------------------------------------------------------------------------
 * k3_xline: cluster of CL CTAs per state, CTA r owns columns [r QC, (r+1) QC) of (y, z);
 * TX threads per (component, column) x-line
 * -------------------------------------------------------------------------------------*/
struct X3Args {
    StepArgs s;                 /* states, ring, coefficients, occupations, slots, qpe, dt ... */
    const void *K;              /* K_yz of every state (TC complex, [2S][N]) */
};

template <typename TC, int CL, int TX_, int HPAD, bool YSF> struct XSmem {
    typedef typename cplx<TC>::t C;
    static constexpr int TX = TX_;
    static constexpr int QC = WTD_L_NYZ / CL;
    static constexpr int LINES = 2 * QC;
    static constexpr int XT = LINES * TX;
    static constexpr int HP = NX + HPAD;                                    /* padded line of H */
    static constexpr size_t tab = (sizeof(LineTab<TC, WTD_L_NMAX>) + 15) / 16 * 16;
    static constexpr size_t hs = (size_t)LINES * HP * sizeof(C);            /* H, then the update, per line */
    /* the state's values per line, where chosen (YSF) and a team of TX > 1 threads shares a
     * line; otherwise each thread reads its points' values from L2/L1 */
    static constexpr bool YS = YSF && TX > 1;
    static constexpr size_t ys = YS ? hs : 0;
    static constexpr size_t scr = (size_t)LINES * team_scratch(NX, TX) * sizeof(C);
    static constexpr size_t red = 80 * sizeof(double);
    static constexpr size_t base = tab + hs + ys + scr + red;
    /* FP64 slabs of the local-term coefficients at this CTA's columns, loaded once per launch
     * (the coefficients are the same for every state): DRE, DIM, V_a, V_b and, with variable
     * mass, N_a, N_b, CJ_a, CJ_b — as many of these as fit beside the rest, in this order;
     * rows of CP doubles, padded so that the 16 lanes of a half warp (4 x-rows of 4 columns)
     * fall on distinct banks */
    static constexpr int CP = QC + 4;
    static constexpr size_t slab = (size_t)NX * CP * sizeof(double);
    /* and slabs in the compute precision of the coefficients the transforms' terms use in that
     * precision anyway — the kinetic coefficient and alpha of each component (AA_a, AA_b, then
     * with variable mass AL_a, AL_b) — rows of CPT (a half warp's 4 x-rows of 8 columns on
     * distinct banks).  Preference, whole pairs of components only: DRE, DIM, V_a, V_b; then the
     * compute-precision slabs; then N_a, N_b, CJ_a, CJ_b. */
    static constexpr int CPT = QC + 8;
    static constexpr size_t tslab = (size_t)NX * CPT * sizeof(TC);
    static constexpr size_t room = base + 64 > WTD_SMEM_MAX ? 0 : WTD_SMEM_MAX - 64 - base;
    static constexpr int NCW = WTD_VAR ? 8 : 4, NTW = WTD_VAR ? 4 : 2;
    static constexpr int NC1 = (int)(room / slab) >= 4 ? 4 : (int)(room / slab) / 2 * 2;
    static constexpr size_t room1 = room - (size_t)NC1 * slab;
    static constexpr int NTS = NC1 < 4 ? 0 : ((int)(room1 / tslab) >= NTW ? NTW : (int)(room1 / tslab) / 2 * 2);
    static constexpr size_t room2 = room1 - (size_t)NTS * tslab;
    static constexpr int NC2 = (NC1 < 4 || NCW == 4) ? 0 : ((int)(room2 / slab) >= 4 ? 4 : (int)(room2 / slab) / 2 * 2);
    static constexpr int NCS = NC1 + NC2;
    static constexpr size_t base2 = base + (size_t)NCS * slab;
    static constexpr size_t bytes = base2 + (size_t)NTS * tslab;
    static constexpr bool ok = WTD_L_NYZ % CL == 0 && XT <= 1024 && XT % 32 == 0 && NX % (TX * TX) == 0;
};

/* the CF_* list entry of coefficient slab k */
__device__ __forceinline__ int xslab_cf(int k)
{
    return k == 0 ? CF_DRE : k == 1 ? CF_DIM : k < 4 ? CF_VA + (k - 2) : k < 6 ? CF_NA + (k - 4) : CF_CJA + (k - 6);
}
/* the CF_* list entry of compute-precision slab k: AA_a, AA_b, then (variable mass) AL_a, AL_b */
__device__ __forceinline__ int xtslab_cf(int k) { return k < 2 ? CF_AA + k : CF_ALA + (k - 2); }

/* Sum over the cluster of one double per thread, in two halves.  cluster_post adds the CTA's
 * values (warp sums, then warp 0 over the warp sums — the order of block_sum), publishes the
 * CTA's partial in its slot and arrives on the cluster barrier without waiting; cluster_collect
 * waits and adds the CTA partials in rank order (the same result on every CTA).  Work placed
 * between the two overlaps the barrier.  Consecutive sums alternate between two slots: the
 * partial of sum k goes where sum k-2 put its own, which every CTA finished reading before it
 * arrived for sum k-1, and it is only written after the wait of sum k-1 — so no partial is
 * overwritten while another CTA may still read it.  The warp-sum array red is rewritten only
 * after the wait of the previous sum, by which time warp 0 has read it. */
template <int CL>
__device__ __forceinline__ void cluster_post(double v, double *red, double *cred, int slot)
{
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if (lane == 0) red[wid] = v;
    __syncthreads();
    if (wid == 0) {
        double s = (lane < nw) ? red[lane] : 0.0;
        s = warp_sum(s);
        if (lane == 0) cred[slot] = s;
    }
    asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
}
template <int CL>
__device__ __forceinline__ double cluster_collect(double *cred, int slot)
{
    namespace cg = cooperative_groups;
    asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
    cg::cluster_group cl = cg::this_cluster();
    double s = 0.0;
#pragma unroll
    for (int r = 0; r < CL; r++) s += *cl.map_shared_rank(cred + slot, r);
    return s;
}

template <typename TY, typename TH, typename TC, int NH, int PASS, bool VAR, bool GRAD, int CL, int TXT, int HPAD, bool YSF>
__global__ void __launch_bounds__(XSmem<TC, CL, TXT, HPAD, YSF>::XT, 1) k3_xline(X3Args xa, const double2 *gtw, const double *gk)
{
    namespace cg = cooperative_groups;
    typedef typename cplx<TC>::t C;
    typedef XSmem<TC, CL, TXT, HPAD, YSF> SM;
    constexpr int N = WTD_NUMEL, NYZ = WTD_L_NYZ, QC = SM::QC, XT = SM::XT, TX = SM::TX, HP = SM::HP;
    constexpr int n1 = NX / TX;
    const StepArgs &a = xa.s;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    LineTab<TC, WTD_L_NMAX> &Tb = *(LineTab<TC, WTD_L_NMAX> *)smem_raw;
    static_assert(sizeof(TY) == sizeof(typename cplx<TC>::t), "states stored in the compute precision");
    /* every region at its XSmem offset: tab | hs | ys | scr | red | slabs */
    C *Hs = (C *)(smem_raw + SM::tab);                                   /* [line][HP] */
    C *Ysm = (C *)(smem_raw + SM::tab + SM::hs);                         /* [line][HP] (YS only) */
    C *Scr = (C *)(smem_raw + SM::tab + SM::hs + SM::ys);                /* [line][team scratch] */
    double *red = (double *)(smem_raw + SM::tab + SM::hs + SM::ys + SM::scr);
    double *cs = (double *)(smem_raw + SM::base);        /* [NCS][NX][CP] coefficient slabs */
    constexpr int NCS = SM::NCS, CP = SM::CP, SL = NX * CP;
    TC *ct = (TC *)(smem_raw + SM::base2);               /* [NTS][NX][CPT] compute-precision slabs */
    constexpr int NTS = SM::NTS, CPT = SM::CPT, STL = NX * CPT;
    __shared__ double cred[2];
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    const int cid = blockIdx.x / CL, ncl = gridDim.x / CL;
    line_tables<TC, WTD_L_NMAX, NX, NY, NZ>(Tb, gtw, gk, WTD_KT);
    const int t = threadIdx.x, line = t / TX, g = t - line * TX;
    const int comp = line / QC, j = line - comp * QC;
    const int q = rank * QC + j;                        /* this team's (y, z) column */
    C *scr = Scr + line * Team<NX, TX>::scratch;
    C *Hl = Hs + line * HP;                             /* this line's H */
    C *Yl = Ysm + line * HP;                            /* this line's state values */
    const C *Yo = Ysm + (comp ? line - QC : line + QC) * HP;   /* the other component's, same column */
    constexpr bool YS = SM::YS;
    const TC sgn = comp ? (TC)-1 : (TC)1;
    TY *Y = (TY *)a.y;
    TY *YO = a.yout ? (TY *)a.yout : Y;
    const C *Kin = (const C *)xa.K;
    const uint64_t pol = l2_policy_keep();
    const size_t SN = (size_t)a.S * N;
    double *ds = a.dslot + (size_t)cid * a.sstride;
    /* this CTA's points of the cluster slot start at zero */
    for (int i = t; i < NX * QC; i += XT) {
        const int x = i / QC, p = x * NYZ + rank * QC + (i - x * QC);
        ds[2 * (size_t)p] = 0.0;
        ds[2 * (size_t)p + 1] = 0.0;
#pragma unroll
        for (int w = 2; w < 12; w++) ds[(size_t)w * N + p] = 0.0;
    }
    for (int k = 0; k < NCS; k++) {
        const double *src = a.cf + (size_t)xslab_cf(k) * N + rank * QC;
        for (int i = t; i < NX * QC; i += XT) {
            const int x = i / QC, jj = i - x * QC;
            cs[k * SL + x * CP + jj] = src[(size_t)x * NYZ + jj];
        }
    }
    for (int k = 0; k < NTS; k++) {
        const double *src = a.cf + (size_t)xtslab_cf(k) * N + rank * QC;
        for (int i = t; i < NX * QC; i += XT) {
            const int x = i / QC, jj = i - x * QC;
            ct[k * STL + x * CPT + jj] = (TC)src[(size_t)x * NYZ + jj];
        }
    }
    __syncthreads();
    int ncalls = 0;   /* cluster sums so far (slot alternation) */

    for (int n = cid; n < a.S; n += ncl) {
        /* L2 prefetch of the next state's inputs at this CTA's columns (one x-row segment per
         * thread: states, K_yz, the ABM slots this pass reads), so that its loads hit L2 */
        {
            const int nn = n + ncl;
            constexpr int NRP = (PASS == 0) ? NH - 1 : (PASS == 1 ? 1 : 0);
            constexpr int NARR = 1 + ((PASS == 1 || PASS == 3 || PASS == 0) ? 1 : 0) + NRP;   /* y, K, ring slots */
            if (nn < a.S && t < NARR * 2 * NX) {
                const int arr = t / (2 * NX), r = t - arr * 2 * NX, c = r / NX, x = r - c * NX;
                const size_t off = (c ? SN : 0) + (size_t)nn * N + (size_t)x * NYZ + rank * QC;
                const void *src;
                size_t bytes;
                if (arr == 0) { src = Y + off; bytes = QC * sizeof(TY); }
                else if (arr == 1 && NARR > NRP + 1) { src = (const C *)xa.K + off; bytes = QC * sizeof(C); }
                else {
                    const int k = arr - (NARR - NRP);
                    const int slot = (PASS == 1) ? NH - 2 : k;
                    src = (const TH *)xa.s.slot[slot] + off;
                    bytes = QC * sizeof(TH);
                }
                prefetch_l2(src, bytes);
            }
        }
        /* tables and coefficients through pointers made opaque per state (ordinary, batched
         * loads inside the iteration, not hoisted out of the state loop) */
        const LineTab<TC, WTD_L_NMAX> &T = *opaque_ptr(&Tb);
        const TC *lapk = T.lapk[0], *dk = T.dk[0];
        const C *tw = T.tw[0];
        const double *cf = opaque_ptr(a.cf);
        const size_t fb = (comp ? SN : 0) + (size_t)n * N;     /* this component of state n */
        const size_t ob = (comp ? 0 : SN) + (size_t)n * N;     /* the other component */
        /* state values at x of this line and of the other component's line at this column */
        auto yown = [&](int x) -> C {
            if (YS) return Yl[x];
            const double2 d = to_d(Y[fb + (size_t)x * NYZ + q]);
            C c; c.x = (TC)d.x; c.y = (TC)d.y;
            return c;
        };
        auto yoth = [&](int x) -> C {
            if (YS) return Yo[x];
            const double2 d = to_d(Y[ob + (size_t)x * NYZ + q]);
            C c; c.x = (TC)d.x; c.y = (TC)d.y;
            return c;
        };
        const bool haveH = (PASS == 1) || (PASS == 3) || (PASS == 0 && !a.fk_given);
        double E = 0.0;
        int eslot = 0;
        /* this line's state values into shared memory (read once from HBM; the local terms of
         * the other component's line read them there too), and K_yz into the line's H */
#pragma unroll 8
        for (int i = 0; i < n1; i++) {
            const int x = g + TX * i, p = x * NYZ + q;
            if (YS) {
                const double2 yd = to_d(Y[fb + p]);
                C c; c.x = (TC)yd.x; c.y = (TC)yd.y;
                Yl[x] = c;
            }
            if (haveH) Hl[x] = Kin[fb + p];
        }
        __syncthreads();
        if (haveH) {
            /* K_yz plus the local terms (pca_kernels.cu:233-391) at this thread's points */
#pragma unroll 2
            for (int i = 0; i < n1; i++) {
                const int x = g + TX * i, p = x * NYZ + q;
                const C cs0 = yown(x), cs1 = yoth(x);
                const C cu = comp ? cs1 : cs0, cv = comp ? cs0 : cs1;
                const double2 u = make_double2((double)cu.x, (double)cu.y), v = make_double2((double)cv.x, (double)cv.y);
                /* this component's coefficients: from the slabs, else from L2 */
                auto co = [&](int k) -> double {
                    return k < NCS ? cs[k * SL + x * CP + j] : ld_ro_keep(cf + (size_t)xslab_cf(k) * N + p, pol);
                };
                const double vs = co(2 + comp), dr = co(0), di = co(1);
                double2 h;
                if (VAR) {
                    const double ns = co(4 + comp), cj = co(6 + comp);
                    if (comp == 0) {
                        h.x = vs * u.x - cj * u.y + (dr * v.x - di * v.y) + ns * u.x;
                        h.y = vs * u.y + cj * u.x + (dr * v.y + di * v.x) + ns * u.y;
                    } else {
                        h.x = -(vs * v.x + cj * v.y) + (dr * u.x + di * u.y) - ns * v.x;
                        h.y = -(vs * v.y - cj * v.x) + (dr * u.y - di * u.x) - ns * v.y;
                    }
                } else {
                    if (comp == 0) {
                        h.x = vs * u.x + (dr * v.x - di * v.y);
                        h.y = vs * u.y + (dr * v.y + di * v.x);
                    } else {
                        h.x = -vs * v.x + (dr * u.x + di * u.y);
                        h.y = -vs * v.y + (dr * u.y - di * u.x);
                    }
                }
                const C k = Hl[x];
                C r; r.x = (TC)(h.x + (double)k.x); r.y = (TC)(h.y + (double)k.y);
                Hl[x] = r;
            }
            /* the x-line part */
            C v[n1], w[n1];
            if (VAR) {
                const int alc = comp ? CF_ALB : CF_ALA;
#pragma unroll
                for (int i = 0; i < n1; i++) {
                    const int p = (g + TX * i) * NYZ + q;
                    const C y = yown(g + TX * i);
                    const TC al = (2 + comp < NTS) ? ct[(2 + comp) * STL + (g + TX * i) * CPT + j]
                                                   : (TC)ld_ro_keep(cf + (size_t)alc * N + p, pol);
                    v[i].x = y.x * al; v[i].y = y.y * al;
                }
                team_fwd<NX, TX>(v, scr, g, tw);
                team_mul_lap<NX, TX>(v, lapk, g);
                team_inv<NX, TX>(v, scr, g, tw);
#pragma unroll
                for (int i = 0; i < n1; i++) {
                    C &h = Hl[g + TX * i];
                    h.x += sgn * (TC)-0.25 * v[i].x; h.y += sgn * (TC)-0.25 * v[i].y;
                }
            }
#pragma unroll
            for (int i = 0; i < n1; i++) v[i] = yown(g + TX * i);
            team_fwd<NX, TX>(v, scr, g, tw);
            if (VAR) {
                const int Ac = comp ? CF_ABX : CF_AAX;
#pragma unroll
                for (int i = 0; i < n1; i++) w[i] = v[i];
                team_mul_d<NX, TX>(w, dk, g);
                team_inv<NX, TX>(w, scr, g, tw);
#pragma unroll
                for (int i = 0; i < n1; i++) {
                    const int x = g + TX * i;
                    const TC A = (TC)ld_ro_keep(cf + (size_t)Ac * N + x * NYZ + q, pol);
                    C &h = Hl[x];
                    h.x += A * w[i].y; h.y += -A * w[i].x;
                }
            }
            team_mul_lap<NX, TX>(v, lapk, g);
            team_inv<NX, TX>(v, scr, g, tw);
            const int aco = comp ? CF_AB : CF_AA;
            double e = 0.0;
#pragma unroll
            for (int i = 0; i < n1; i++) {
                const int x = g + TX * i, p = x * NYZ + q;
                const TC ac = sgn * ((comp < NTS) ? ct[comp * STL + x * CPT + j] : (TC)ld_ro_keep(cf + (size_t)aco * N + p, pol));
                C h = Hl[x];
                h.x += ac * v[i].x; h.y += ac * v[i].y;
                Hl[x] = h;
                const C y = yown(x);
                e += (double)y.x * (double)h.x + (double)y.y * (double)h.y;
            }
            eslot = ncalls & 1;
            ncalls++;
            cluster_post<CL>(e, red, cred, eslot);
        }
        /* the ABM inputs of this thread's points, loaded while the cluster sum of <H> completes:
         * the first NRP history slots this pass reads (none where a thread owns more than 8
         * points of a line: they would not stay in registers) */
        constexpr int NR = (PASS == 0) ? NH - 1 : (PASS == 1 ? 1 : 0);
        constexpr int NRP = n1 > 8 ? 0 : (PASS == 0) ? (sizeof(TH) == 8 ? 2 : 1) : (PASS == 1 ? 1 : 0);
        auto ring = [&](int k) -> const TH * { return (const TH *)xa.s.slot[PASS == 1 ? NH - 2 : k]; };
        TH frr[NRP > 0 ? NRP : 1][NRP > 0 ? n1 : 1];
        if constexpr (NRP > 0) {
#pragma unroll
            for (int i = 0; i < n1; i++) {
                const size_t gi = fb + (size_t)(g + TX * i) * NYZ + q;
#pragma unroll
                for (int k = 0; k < NRP; k++) frr[k][i] = ld_stream(ring(k) + gi);
            }
        }
        if (haveH) {
            E = cluster_collect<CL>(cred, eslot) * WTD_DV;
            if (t == 0 && rank == 0) a.qpe[n] = E;
        }
        if (PASS == 3) {
#pragma unroll 2
            for (int i = 0; i < n1; i++) {
                const int x = g + TX * i;
                const size_t gi = fb + x * NYZ + q;
                const C yc = yown(x);
                const double2 y0 = make_double2((double)yc.x, (double)yc.y);
                const C h = Hl[x];
                ((TH *)xa.s.slot[NH - 1])[gi] = from_d<TH>(make_double2((double)h.x - E * y0.x, (double)h.y - E * y0.y));
            }
            __syncthreads();
            continue;
        }
        /* ---- ABM update of this thread's points, unnormalised into H (fully unrolled where
         * the preloaded history words index frr by i; two points at a time otherwise) ---- */
        double nrm = 0.0;
        constexpr int ABMU = NRP > 0 ? n1 : 2;
#pragma unroll ABMU
        for (int i = 0; i < n1; i++) {
            const int x = g + TX * i;
            const size_t gi = fb + x * NYZ + q;
            const C yc = yown(x);
            const double2 y0 = make_double2((double)yc.x, (double)yc.y);
            double2 fr[NR > 0 ? NR : 1], fkg = make_double2(0.0, 0.0);
#pragma unroll
            for (int k = 0; k < NR; k++) fr[k] = to_d(k < NRP ? frr[k < NRP ? k : 0][NRP > 0 ? i : 0] : ld_stream(ring(k) + gi));
            if (PASS == 0 && !haveH) fkg = to_d(ld_stream((const TH *)xa.s.slot[NH - 1] + gi));
            double2 fk = make_double2(0.0, 0.0);
            if (PASS != 2) {
                if (haveH) {
                    const C h = Hl[x];
                    fk.x = (double)h.x - E * y0.x;
                    fk.y = (double)h.y - E * y0.y;
                } else {
                    fk = fkg;
                }
            }
            double2 out;
            if (PASS == 2) {
                out = y0;
            } else if (PASS == 0) {
                typedef Abm<NH> A;
                double2 sb = make_double2(fk.x * A::b(0), fk.y * A::b(0));
                double2 sa = make_double2(fk.x * A::a(0), fk.y * A::a(0));
#pragma unroll
                for (int k = 1; k < NH; k++) {
                    const double2 fj = fr[k - 1];
                    sb.x += fj.x * A::b(k); sb.y += fj.y * A::b(k);
                    if (k < A::na) { sa.x += fj.x * A::a(k); sa.y += fj.y * A::a(k); }
                }
                out.x = y0.x + a.dt * sb.y; out.y = y0.y - a.dt * sb.x;
                const double2 P = make_double2(y0.x + a.dt * sa.y, y0.y - a.dt * sa.x);
                if (haveH) st_stream((TH *)xa.s.slot[NH - 1] + gi, from_d<TH>(fk));
                st_stream((TH *)xa.s.slot[NH - 2] + gi, from_d<TH>(P));
            } else {
                const double2 P = fr[0];
                const double cc = Abm<NH>::c;
                out.x = a.dt * fk.y * cc + P.x;
                out.y = -a.dt * fk.x * cc + P.y;
            }
            nrm += out.x * out.x + out.y * out.y;
            C r; r.x = (TC)out.x; r.y = (TC)out.y;
            Hl[x] = r;
        }
        const int nslot = ncalls & 1;
        ncalls++;
        cluster_post<CL>(nrm, red, cred, nslot);
        const double nrm_tot = sqrt(cluster_collect<CL>(cred, nslot) * WTD_DV);
        const double cinv = 1.0 / nrm_tot;
        if (a.nrm_out && t == 0 && rank == 0) a.nrm_out[n] = nrm_tot;
        /* ---- normalise, store; the stored values are what the densities see ---- */
#pragma unroll 2
        for (int i = 0; i < n1; i++) {
            const int x = g + TX * i;
            const size_t gi = fb + x * NYZ + q;
            const C h = Hl[x];
            const TY s = from_d<TY>(make_double2((double)h.x * cinv, (double)h.y * cinv));
            st_stream(YO + gi, s);
            const double2 sd = to_d(s);
            C r; r.x = (TC)sd.x; r.y = (TC)sd.y;
            Hl[x] = r;
        }
        __syncthreads();
        const double f = a.occ[n], wgt = a.wcnt[n];
        for (int i = t; i < NX * QC; i += XT) {
            const int x = i / QC, jj = i - x * QC;
            const int p = x * NYZ + rank * QC + jj;
            const C hu = Hs[jj * HP + x], hv = Hs[(QC + jj) * HP + x];
            dens_limited_red(ds, p, N, make_double2((double)hu.x, (double)hu.y), make_double2((double)hv.x, (double)hv.y), f, wgt,
                             pol);
        }
        if (GRAD) {
            /* x-parts of tau_tmp = Re[psi* lap psi] and j_x = Im[psi* d_x psi] (pca_dens.cu:41-108) */
            const double fw = (comp == 0 ? f : (1.0 - f)) * wgt;
            const double jsgn = comp == 0 ? 1.0 : -1.0;
            const int tau_q = comp == 0 ? 3 : 8, j_q = comp == 0 ? 4 : 9;
            C v[n1], w[n1];
#pragma unroll
            for (int i = 0; i < n1; i++) v[i] = Hl[g + TX * i];
            team_fwd<NX, TX>(v, scr, g, tw);
#pragma unroll
            for (int i = 0; i < n1; i++) w[i] = v[i];
            team_mul_d<NX, TX>(w, dk, g);
            team_inv<NX, TX>(w, scr, g, tw);
            team_mul_lap<NX, TX>(v, lapk, g);
            team_inv<NX, TX>(v, scr, g, tw);
#pragma unroll
            for (int i = 0; i < n1; i++) {
                const int x = g + TX * i, p = x * NYZ + q;
                const C s = Hl[x];
                red_keep(ds + (size_t)j_q * N + p, jsgn * ((double)s.x * (double)w[i].y - (double)s.y * (double)w[i].x) * fw, pol);
                red_keep(ds + (size_t)tau_q * N + p, ((double)s.x * (double)v[i].x + (double)s.y * (double)v[i].y) * fw, pol);
            }
        }
        __syncthreads();
    }
    /* no CTA leaves while another may still read its cluster-sum slots */
    cluster.sync();
}

/* one axis of the density part for one team: j_d and the d-part of tau_tmp of the line */
template <int n, int T, typename TC>
__device__ __forceinline__ void plane_dens_axis(const typename cplx<TC>::t *P, typename cplx<TC>::t *scr,
                                               const LineTab<TC, WTD_L_NMAX> &Tb, int ax, int g, int line,
                                               double *acc, double fw, double jsgn)
{
    typedef typename cplx<TC>::t C;
    constexpr int n1 = n / T, PITCH = PlaneGeo::PITCH, NYZ = WTD_L_NYZ;
    const bool yl = ax == 1;
    auto at = [&](int i) -> int { const int c = g + T * i; return yl ? c * PITCH + line : line * PITCH + c; };
    auto ai = [&](int i) -> int { const int c = g + T * i; return yl ? c * NZ + line : line * NZ + c; };
    const TC *lapk = Tb.lapk[ax], *dk = Tb.dk[ax];
    const C *tw = Tb.tw[ax];
    double *aj = acc + (size_t)ax * NYZ;
    C v[n1], w[n1];
#pragma unroll
    for (int i = 0; i < n1; i++) v[i] = P[at(i)];
    team_fwd<n, T>(v, scr, g, tw);
#pragma unroll
    for (int i = 0; i < n1; i++) w[i] = v[i];
    team_mul_d<n, T>(w, dk, g);
    team_inv<n, T>(w, scr, g, tw);
    team_mul_lap<n, T>(v, lapk, g);
    team_inv<n, T>(v, scr, g, tw);
    /* accumulators read before any is written (half a line at a time), so that the shared-memory
     * round trips overlap instead of forming one chain */
    constexpr int HB = n1 > 4 ? n1 / 2 : n1;
#pragma unroll
    for (int i0 = 0; i0 < n1; i0 += HB) {
        double tj[HB], ta[HB];
#pragma unroll
        for (int i = 0; i < HB; i++) { tj[i] = aj[ai(i0 + i)]; ta[i] = acc[ai(i0 + i)]; }
#pragma unroll
        for (int i = 0; i < HB; i++) {
            const C s = P[at(i0 + i)];
            tj[i] += jsgn * ((double)s.x * (double)w[i0 + i].y - (double)s.y * (double)w[i0 + i].x) * fw;
            ta[i] += ((double)s.x * (double)v[i0 + i].x + (double)s.y * (double)v[i0 + i].y) * fw;
        }
#pragma unroll
        for (int i = 0; i < HB; i++) { aj[ai(i0 + i)] = tj[i]; acc[ai(i0 + i)] = ta[i]; }
    }
}

/* ---------------------------------------------------------------------------------------
 * k3_plane_dens: (y, z) parts of tau and j of the updated states.  blockIdx.x = (comp, x,
 * chunk g); the CTA sums the states g, g + G, ... and writes slot g of its plane's points:
 * tau_tmp and j_y, j_z of its component, zeros in the words of this slot that the x-line pass
 * fills in its own slots (nu, rho, j_x).
 * -------------------------------------------------------------------------------------*/
template <typename TY, typename TC>
__global__ void __launch_bounds__(PlaneGeo::PT) k3_plane_dens(const TY *__restrict__ Y, const double *occ, const double *wcnt,
                                                             int S, int G, double *slots, size_t sstride, const double2 *gtw,
                                                             const double *gk)
{
    typedef typename cplx<TC>::t C;
    typedef PlaneSmem<TC> SM;
    typedef PlaneGeo PG;
    constexpr int N = WTD_NUMEL, NYZ = WTD_L_NYZ, PT = PG::PT, PITCH = PG::PITCH;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    LineTab<TC, WTD_L_NMAX> &Tb = *(LineTab<TC, WTD_L_NMAX> *)smem_raw;
    C *P = (C *)(smem_raw + SM::tab);
    C *Sc = P + (NY) * PITCH;
    double *acc = (double *)(smem_raw + SM::tab + SM::plane + SM::scr);   /* [3][NYZ]: tau, j_y, j_z */
    line_tables<TC, WTD_L_NMAX, NX, NY, NZ>(Tb, gtw, gk, WTD_KT);
    const int t = threadIdx.x;
    const int gch = blockIdx.x % G, rest = blockIdx.x / G;
    const int x = rest % NX, comp = rest / NX;
    for (int i = t; i < 3 * NYZ; i += PT) acc[i] = 0.0;
    __syncthreads();
    const double jsgn = comp == 0 ? 1.0 : -1.0;
    for (int n = gch; n < S; n += G) {
        const double f = occ[n], w = wcnt[n];
        const double fw = (comp == 0 ? f : (1.0 - f)) * w;
        const size_t base = ((size_t)comp * S + n) * N + (size_t)x * NYZ;
        const LineTab<TC, WTD_L_NMAX> &T = *opaque_ptr(&Tb);
        if (t == 0 && n + G < S) prefetch_l2(Y + base + (size_t)G * N, (size_t)NYZ * sizeof(TY));
        for (int i = t; i < NYZ; i += PT) {
            const double2 a = to_d(Y[base + i]);
            C c; c.x = (TC)a.x; c.y = (TC)a.y;
            P[(i / NZ) * PITCH + (i % NZ)] = c;
        }
        __syncthreads();
        if (t < PG::AY) {
            const int line = t / PG::TY, g = t - line * PG::TY;
            plane_dens_axis<NY, PG::TY, TC>(P, Sc + line * Team<NY, PG::TY>::scratch, T, 1, g, line, acc, fw, jsgn);
        }
        __syncthreads();
        if (t < PG::AZ) {
            const int line = t / PG::TZ, g = t - line * PG::TZ;
            plane_dens_axis<NZ, PG::TZ, TC>(P, Sc + line * Team<NZ, PG::TZ>::scratch, T, 2, g, line, acc, fw, jsgn);
        }
        __syncthreads();
    }
    /* slot gch: this plane's words of this component */
    double *ds = slots + (size_t)gch * sstride;
    const int pb = x * NYZ;
    const int tau_q = comp == 0 ? 3 : 8, j_q = comp == 0 ? 4 : 9;
    for (int i = t; i < NYZ; i += PT) {
        const int p = pb + i;
        ds[(size_t)tau_q * N + p] = acc[i];
        ds[(size_t)(j_q + 1) * N + p] = acc[NYZ + i];
        ds[(size_t)(j_q + 2) * N + p] = acc[2 * NYZ + i];
        ds[(size_t)j_q * N + p] = 0.0;
        if (comp == 0) {
            ds[2 * (size_t)p] = 0.0;
            ds[2 * (size_t)p + 1] = 0.0;
            ds[2 * (size_t)N + p] = 0.0;
        } else {
            ds[7 * (size_t)N + p] = 0.0;
        }
    }
}

#undef CFP
#endif /* CODEDIM == 3 */
#endif
