/*
 * Checkpoint files in the reference's layout (hpc-engine/tdwslda_checkpoint.c), so that a run
 * can restart from a checkpoint the reference wrote (inittype 5) and the reference can restart
 * from one written here.
 *
 * One file <dir>/checkpoint_<g> per IO group g of `howmany` consecutive ranks
 * (MPI_NP_PER_IO_GROUP, pca.c:65-67).  Every rank writes its own blocks at fixed offsets;
 * the first rank of a group also writes the header and the potentials.  Layout, all
 * little-endian and unaligned:
 *
 *   header   t0, mu_a, mu_b, ec, kF (f64), nwf (i32), eF, Effg, beta (f64)       68 bytes
 *   E_n      per rank of the group: `slot` f64 (the rank's nwfip energies first)
 *   k_perp   2D: k_z; 1D: k_y then k_z, each as E_n                              (not in 3D)
 *   states   per rank: 2 slot N complex ([u_0..u_{nwfip-1}, v_0..v_{nwfip-1}] first)
 *   f_1..f_q the ABM history (q = 3, 4, 5 for AB3AM4, AB4AM5, AB5AM5), each as the states
 *   pots     12 N f64, the potentials
 *
 * with slot = nwfip + (rank < nwf % nranks ? 0 : 1) = nwf / nranks + 1 for every rank
 * (tdwslda_checkpoint.c:132-140) and nwfip the rank's state count (getnwfip, pca_utils.c:660).
 * The energies, not the occupations, are stored; loading recomputes f = fbeta(E_n, beta)
 * (pca.c:830, pca_uniform.h:70-76).  1D degeneracy counts are not stored (the reference
 * recomputes them from k_y, k_z, ccpca.c:546): the caller passes the ones the run started with.
 */
#ifndef WTD_CHECKPOINT_CUH
#define WTD_CHECKPOINT_CUH

#include <fcntl.h>
#include <unistd.h>

struct CkLayout {
    int nwfip, slot, ip, gsize, group;
    size_t en, kp[2], arr[6], pots; /* arr[0]: states, arr[1..q]: f_1..f_q */
};

/* offsets of one rank's blocks in its group's file (tdwslda_checkpoint.c:252-356) */
static void ck_layout(int nwf, int rank, int nranks, int howmany, CkLayout *L)
{
    constexpr size_t N = WTD_NUMEL;
    L->nwfip = nwf / nranks + (rank < nwf % nranks ? 1 : 0);
    L->slot = L->nwfip + (rank < nwf % nranks ? 0 : 1);
    L->group = rank / howmany;
    L->ip = rank - L->group * howmany;
    L->gsize = nranks - L->group * howmany < howmany ? nranks - L->group * howmany : howmany;
    size_t s0 = 5 * sizeof(double) + sizeof(int) + 3 * sizeof(double);
    const size_t vb = sizeof(double) * (size_t)L->slot;
    L->en = s0 + vb * L->ip;
    s0 += vb * L->gsize;
    L->kp[0] = L->kp[1] = 0;
    if (CODEDIM <= 2) { L->kp[0] = s0 + vb * L->ip; s0 += vb * L->gsize; }
    if (CODEDIM == 1) { L->kp[1] = s0 + vb * L->ip; s0 += vb * L->gsize; }
    const size_t ab = (size_t)2 * L->slot * N * 2 * sizeof(double);
    for (int a = 0; a <= WTD_NHIST; a++) { L->arr[a] = s0 + ab * L->ip; s0 += ab * L->gsize; }
    L->pots = s0;
}

static void ck_path(char *out, size_t n, const char *dir, int group)
{
    snprintf(out, n, "%s/checkpoint_%d", dir, group);
}

static int ck_pio(int fd, void *buf, size_t bytes, size_t off, bool wr)
{
    char *p = (char *)buf;
    while (bytes > 0) {
        ssize_t r = wr ? pwrite(fd, p, bytes, (off_t)off) : pread(fd, p, bytes, (off_t)off);
        if (r <= 0) return WTD_ERR_IO;
        p += r; off += (size_t)r; bytes -= (size_t)r;
    }
    return WTD_OK;
}

static int ck_header(int fd, wtd_checkpoint_info *info, bool wr)
{
    unsigned char h[68];
    double d[8];
    int nwf = 0;
    if (wr) {
        d[0] = info->t0; d[1] = info->mu_a; d[2] = info->mu_b; d[3] = info->ec; d[4] = info->kF;
        d[5] = info->eF; d[6] = info->Effg; d[7] = info->beta; nwf = info->nwf;
        memcpy(h, d, 40); memcpy(h + 40, &nwf, 4); memcpy(h + 44, d + 5, 24);
        return ck_pio(fd, h, 68, 0, true);
    }
    WTD_TRY(ck_pio(fd, h, 68, 0, false));
    memcpy(d, h, 40); memcpy(&nwf, h + 40, 4); memcpy(d + 5, h + 44, 24);
    info->t0 = d[0]; info->mu_a = d[1]; info->mu_b = d[2]; info->ec = d[3]; info->kF = d[4];
    info->eF = d[5]; info->Effg = d[6]; info->beta = d[7]; info->nwf = nwf;
    return WTD_OK;
}

/* occupation of energy E at inverse temperature beta (pca_uniform.h:70-76) */
static double ck_fbeta(double E, double beta)
{
    const double bE = beta * E;
    if (bE > 50.) return 0.0;
    if (bE < -50.) return 1.0;
    return 1.0 / (exp(bE) + 1.0);
}

extern "C" int wtd_checkpoint_info_read(const char *dir, int rank, int howmany, wtd_checkpoint_info *info)
{
    if (!dir || !info || rank < 0 || howmany < 1) return WTD_ERR_ARG;
    char path[4096];
    ck_path(path, sizeof(path), dir, rank / howmany);
    int fd = open(path, O_RDONLY);
    if (fd < 0) return WTD_ERR_IO;
    const int r = ck_header(fd, info, false);
    close(fd);
    if (r == WTD_OK && info->nwf <= 0) return WTD_ERR_IO;
    return r;
}

extern "C" int wtd_checkpoint_save(wtd_ctx *c, const char *dir, int rank, int nranks, int howmany,
                                   const wtd_checkpoint_info *info, const double *En, const double *kperp)
{
    if (!c || !dir || !info || !En || rank < 0 || nranks < 1 || rank >= nranks || howmany < 1) return WTD_ERR_ARG;
    if ((CODEDIM <= 2) && !kperp) return WTD_ERR_ARG;
    CkLayout L;
    ck_layout(info->nwf, rank, nranks, howmany, &L);
    if (L.nwfip != c->S) return WTD_ERR_ARG;
    WTD_CU(cudaSetDevice(c->dev));
    WTD_TRY(ensure_fk(c)); /* f_1 is formed on demand (the reference's end-of-step H psi) */
    char path[4096];
    ck_path(path, sizeof(path), dir, L.group);
    int fd = open(path, O_WRONLY | O_CREAT, 0644);
    if (fd < 0) return WTD_ERR_IO;
    const size_t n2 = (size_t)2 * c->S * WTD_NUMEL;
    std::vector<double> buf(2 * n2);
    int r = WTD_OK;
    wtd_checkpoint_info hdr = *info;
    if (L.ip == 0) r = ck_header(fd, &hdr, true);
    if (r == WTD_OK) r = ck_pio(fd, (void *)En, sizeof(double) * c->S, L.en, true);
    for (int k = 0; k < 2 && r == WTD_OK; k++)
        if (L.kp[k]) r = ck_pio(fd, (void *)(kperp + (size_t)k * c->S), sizeof(double) * c->S, L.kp[k], true);
    if (r == WTD_OK) r = wtd_download_states(c, buf.data());
    if (r == WTD_OK) r = ck_pio(fd, buf.data(), sizeof(double) * 2 * n2, L.arr[0], true);
    for (int h = 0; h < WTD_NHIST && r == WTD_OK; h++) {
        r = wtd_download_history(c, h, buf.data());
        if (r == WTD_OK) r = ck_pio(fd, buf.data(), sizeof(double) * 2 * n2, L.arr[1 + h], true);
    }
    if (r == WTD_OK && L.ip == 0) {
        std::vector<double> p(12 * (size_t)WTD_NUMEL);
        r = wtd_download_potentials(c, p.data());
        if (r == WTD_OK) r = ck_pio(fd, p.data(), sizeof(double) * p.size(), L.pots, true);
    }
    if (close(fd) != 0 && r == WTD_OK) r = WTD_ERR_IO;
    return r;
}

extern "C" int wtd_checkpoint_load(wtd_ctx *c, const char *dir, int rank, int nranks, int howmany, const int *cnt,
                                   wtd_checkpoint_info *info, double *En, double *kperp)
{
    if (!c || !dir || rank < 0 || nranks < 1 || rank >= nranks || howmany < 1) return WTD_ERR_ARG;
    wtd_checkpoint_info hdr;
    WTD_TRY(wtd_checkpoint_info_read(dir, rank, howmany, &hdr));
    CkLayout L;
    ck_layout(hdr.nwf, rank, nranks, howmany, &L);
    if (L.nwfip != c->S) return WTD_ERR_ARG;
    WTD_CU(cudaSetDevice(c->dev));
    char path[4096];
    ck_path(path, sizeof(path), dir, L.group);
    int fd = open(path, O_RDONLY);
    if (fd < 0) return WTD_ERR_IO;
    const int S = c->S;
    const size_t n2 = (size_t)2 * S * WTD_NUMEL;
    std::vector<double> buf(2 * n2), en(S), kp(2 * (size_t)S, 0.0), occ(S);
    int r = ck_pio(fd, en.data(), sizeof(double) * S, L.en, false);
    for (int k = 0; k < 2 && r == WTD_OK; k++)
        if (L.kp[k]) r = ck_pio(fd, kp.data() + (size_t)k * S, sizeof(double) * S, L.kp[k], false);
    /* the run restarts at time index 0 of the loaded time, history as stored (pca.c:781-830) */
    c->it = 0;
    c->head = 0;
    c->qfsw = 0.0;
    if (r == WTD_OK) r = ck_pio(fd, buf.data(), sizeof(double) * 2 * n2, L.arr[0], false);
    if (r == WTD_OK) r = wtd_upload_states(c, buf.data());
    for (int h = 0; h < WTD_NHIST && r == WTD_OK; h++) {
        r = ck_pio(fd, buf.data(), sizeof(double) * 2 * n2, L.arr[1 + h], false);
        if (r == WTD_OK) r = wtd_upload_history(c, h, buf.data());
    }
    if (r == WTD_OK) {
        std::vector<double> p(12 * (size_t)WTD_NUMEL);
        r = ck_pio(fd, p.data(), sizeof(double) * p.size(), L.pots, false);
        if (r == WTD_OK) r = wtd_upload_potentials(c, p.data());
    }
    close(fd);
    WTD_TRY(r);
    for (int n = 0; n < S; n++) occ[n] = ck_fbeta(en[n], hdr.beta);
    const double *kky = CODEDIM == 1 ? kp.data() : nullptr;
    const double *kkz = CODEDIM == 2 ? kp.data() : (CODEDIM == 1 ? kp.data() + S : nullptr);
    WTD_TRY(wtd_upload_occupations(c, occ.data(), kky, kkz, cnt));
    /* the restart's measurement (pca.c:939-958): normalise and densities, history kept */
    c->fk_given = 1;
    if (c->staged) {
        WTD_TRY(staged_initial(c));
    } else if (c->line) {
        WTD_TRY(line_initial(c));
    } else {
        WTD_TRY(run_pass(c, 2, true));
        WTD_TRY(after_pass(c, true, -1));
    }
    WTD_TRY(wtd_cuerr(cudaStreamSynchronize(c->st)));
    if (info) *info = hdr;
    if (En) memcpy(En, en.data(), sizeof(double) * S);
    if (kperp) memcpy(kperp, kp.data(), sizeof(double) * (CODEDIM == 1 ? 2 * (size_t)S : (size_t)S));
    return WTD_OK;
}

#endif
