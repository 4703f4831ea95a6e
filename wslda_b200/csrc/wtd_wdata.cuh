/*
 * Measurements in the W-data format the reference's TD codes write (hpc-engine/wslda_writevars.c,
 * lib/wdata), so the reference's post-processing and visualisation tools read runs made here.
 *
 * A data set is <prefix>.wtxt (text metadata: lattice, datadim, prefix, cycles, t0, dt, the
 * variables with their types, links between spin-symmetric twins, constants) and one
 * <prefix>_<var>.wdat per variable holding the cycles back to back as raw little-endian f64 (f32
 * for writeprec f).  Variables follow the input's `writevar` tags the way create_wdata_metadata
 * expands them (wslda_writevars.c:103-246):
 *
 *   rho/density -> rho_a, rho_b      j/current -> j_a, j_b (vector: x, y, z)   tau -> tau_a, tau_b
 *   V -> V_a, V_b (mean field minus V_ext)   V_ext -> V_ext_a, V_ext_b   velocity_ext -> _a, _b
 *   delta, delta_ext, nu (complex)          alpha -> alpha_a, alpha_b   A -> A_a, A_b (vector)
 *
 * with the b twin written as a link to the a variable in spin-symmetric runs.  The constants
 * are kF, eF, mu_a, mu_b (pca.c:1026-1030).  Each wtd_wdata_write appends one cycle of every
 * variable from the current densities and potentials at the context's time index and rewrites
 * the metadata (write_measurments, wslda_writevars.c:298-470; pca.c:1044-1046, 1628-1630).
 */
#ifndef WTD_WDATA_CUH
#define WTD_WDATA_CUH

#include <string>
#include <ctime>

namespace wdata_out {

enum Src { RHO_A, RHO_B, J_A, J_B, TAU_A, TAU_B, V_A, V_B, VEXT_A, VEXT_B, VELEXT_A, VELEXT_B, DELTA, DELTA_EXT, NU,
           ALPHA_A, ALPHA_B, A_A, A_B };

struct Var {
    std::string name, type;
    int src, comps; /* doubles per point: 1 real, 2 complex, 3 vector */
};

struct Set {
    std::string prefix;
    int datadim, cycles;
    double t0, dt;
    bool fprec;
    std::vector<Var> vars;
    std::vector<std::pair<std::string, std::string>> links;
};

static void free_set(void *p) { delete (Set *)p; }

/* one writevar tag -> its variables (wslda_writevars.c:143-244) */
static bool add_tag(Set *s, const std::string &tag, bool sym)
{
    const char *rt = s->fprec ? "real4" : "real", *ct = s->fprec ? "complex8" : "complex",
               *vt = s->fprec ? "vector4" : "vector";
    auto pair = [&](const char *a, const char *b, const char *type, int sa, int sb, int comps) {
        s->vars.push_back({a, type, sa, comps});
        if (!sym) s->vars.push_back({b, type, sb, comps});
        else s->links.push_back({b, a});
    };
    if (tag == "density" || tag == "rho") pair("rho_a", "rho_b", rt, RHO_A, RHO_B, 1);
    else if (tag == "current" || tag == "j") pair("j_a", "j_b", vt, J_A, J_B, 3);
    else if (tag == "tau") pair("tau_a", "tau_b", rt, TAU_A, TAU_B, 1);
    else if (tag == "V") pair("V_a", "V_b", rt, V_A, V_B, 1);
    else if (tag == "V_ext") pair("V_ext_a", "V_ext_b", rt, VEXT_A, VEXT_B, 1);
    else if (tag == "velocity_ext") pair("velocity_ext_a", "velocity_ext_b", vt, VELEXT_A, VELEXT_B, 3);
    else if (tag == "delta") s->vars.push_back({"delta", ct, DELTA, 2});
    else if (tag == "delta_ext") s->vars.push_back({"delta_ext", ct, DELTA_EXT, 2});
    else if (tag == "nu") s->vars.push_back({"nu", ct, NU, 2});
    else if (tag == "alpha") pair("alpha_a", "alpha_b", rt, ALPHA_A, ALPHA_B, 1);
    else if (tag == "A") pair("A_a", "A_b", vt, A_A, A_B, 3);
    else return false;
    return true;
}

/* the metadata text (wdata_print_metadata, lib/wdata/c/wdata.c:495-564) */
static int write_meta(const Set *s)
{
    std::string path = s->prefix + ".wtxt";
    FILE *f = fopen(path.c_str(), "w");
    if (!f) return WTD_ERR_IO;
    char stamp[32];
    time_t now = time(nullptr);
    strftime(stamp, sizeof(stamp), "%x-%X", localtime(&now));
    fprintf(f, "# Generated by td-wslda-%dd (wslda_b200) [%s]\n\n", CODEDIM, stamp);
    fprintf(f, "# W-DATA 0.3.0\n");
    fprintf(f, "# More information about the WData format see: https://gitlab.fizyka.pw.edu.pl/wtools/wdata/-/wikis/home\n");
    fprintf(f, "nx %24d   # lattice\n", NX);
    fprintf(f, "ny %24d   # lattice\n", NY);
    fprintf(f, "nz %24d   # lattice\n", NZ);
    fprintf(f, "dx %24g   # spacing\n", (double)DX);
    fprintf(f, "dy %24g   # spacing\n", (double)DY);
    fprintf(f, "dz %24g   # spacing\n", (double)DZ);
    fprintf(f, "datadim %19d   # dimension of block size: 1=nx, 2=nx*ny, 3=nx*ny*nz\n", s->datadim);
    if (s->prefix.size() > 20)
        fprintf(f, "prefix %s   # prefix for files belonging to this data set`\n", s->prefix.c_str());
    else
        fprintf(f, "prefix %20s   # prefix for files belonging to this data set`\n", s->prefix.c_str());
    fprintf(f, "cycles %20d   # number of cycles (measurements)\n", s->cycles);
    fprintf(f, "t0 %24g   # time value for the first cycle\n", s->t0);
    fprintf(f, "dt %24g   # time interval between cycles\n", s->dt);
    fprintf(f, "\n# variables\n");
    fprintf(f, "# tag                  name                    type                    unit                  format\n");
    for (const Var &v : s->vars) fprintf(f, "var%24s%24s%24s%24s\n", v.name.c_str(), v.type.c_str(), "none", "wdat");
    if (!s->links.empty()) {
        fprintf(f, "\n# links\n");
        fprintf(f, "# tag                  name                 link-to\n");
        for (const auto &l : s->links) fprintf(f, "link%23s%24s\n", l.first.c_str(), l.second.c_str());
    }
    fprintf(f, "\n# consts\n");
    fprintf(f, "# tag                  name                   value                    unit\n");
    const char *cn[4] = {"kF", "eF", "mu_a", "mu_b"};
    const double cvals[4] = {hc_kF, hc_eF, hc_mu_a, hc_mu_b};
    for (int k = 0; k < 4; k++) fprintf(f, "const%22s%24g%24s\n", cn[k], cvals[k], "none");
    fprintf(f, "\n");
    return fclose(f) == 0 ? WTD_OK : WTD_ERR_IO;
}

} // namespace wdata_out

extern "C" int wtd_wdata_begin(wtd_ctx *c, const char *prefix, const char *vars, double t0, double dt_cycle,
                               int float_prec)
{
    using namespace wdata_out;
    if (!c || !prefix || !*prefix) return WTD_ERR_ARG;
    Set *s = new Set();
    s->prefix = prefix;
    s->datadim = CODEDIM;
    s->cycles = 0;
    s->t0 = t0;
    s->dt = dt_cycle;
    s->fprec = float_prec != 0;
#ifdef SPINSYMMETRY_MODE
    const bool sym = true;
#else
    const bool sym = false;
#endif
    std::string list = (vars && *vars) ? vars : "rho delta j"; /* the input's default (pca_utils.c:560-565) */
    for (char &ch : list) if (ch == ',' || ch == ';' || ch == '\t') ch = ' ';
    size_t i = 0;
    while (i < list.size()) {
        while (i < list.size() && list[i] == ' ') i++;
        size_t j = i;
        while (j < list.size() && list[j] != ' ') j++;
        if (j > i && !add_tag(s, list.substr(i, j - i), sym)) { delete s; return WTD_ERR_ARG; }
        i = j;
    }
    /* a fresh data set (clear_files, wslda_writevars.c:253-260) */
    for (const Var &v : s->vars) remove((s->prefix + "_" + v.name + ".wdat").c_str());
    const int r = write_meta(s);
    if (r != WTD_OK) { delete s; return r; }
    if (c->wdata && c->wdata_free) c->wdata_free(c->wdata);
    c->wdata = s;
    c->wdata_free = free_set;
    return WTD_OK;
}

extern "C" int wtd_wdata_write(wtd_ctx *c)
{
    using namespace wdata_out;
    if (!c) return WTD_ERR_ARG;
    Set *s = (Set *)c->wdata;
    if (!s) return WTD_ERR_STATE;
    WTD_CU(cudaSetDevice(c->dev));
    constexpr size_t N = WTD_NUMEL;
    std::vector<double> dens(12 * N), pots(12 * N), ext(3 * N);
    WTD_TRY(wtd_download_densities(c, dens.data()));
    WTD_TRY(wtd_download_potentials(c, pots.data()));
    const int it = c->it;
    for (const Var &v : s->vars) {
        const double *src = nullptr;
        switch (v.src) {
        case RHO_A: src = &dens[2 * N]; break;
        case RHO_B: src = &dens[7 * N]; break;
        case TAU_A: src = &dens[3 * N]; break;
        case TAU_B: src = &dens[8 * N]; break;
        case J_A: src = &dens[4 * N]; break;
        case J_B: src = &dens[9 * N]; break;
        case NU: src = &dens[0]; break;
        case DELTA: src = &pots[2 * N]; break;
        case ALPHA_A: src = &pots[4 * N]; break;
        case ALPHA_B: src = &pots[5 * N]; break;
        case A_A: src = &pots[6 * N]; break;
        case A_B: src = &pots[9 * N]; break;
        case V_A: case V_B: case VEXT_A: case VEXT_B: {
            const int spin = (v.src == V_A || v.src == VEXT_A) ? SPINA : SPINB;
            if (get_v_ext(CODEDIM, spin, it, ext.data())) return WTD_ERR_CUDA;
            if (v.src == V_A || v.src == V_B) {
                /* the mean field without the external potential (wslda_writevars.c:352-370) */
                const double *V = &pots[(spin == SPINA ? 0 : 1) * N];
                for (size_t p = 0; p < N; p++) ext[p] = V[p] - ext[p];
            }
            src = ext.data();
            break;
        }
        case VELEXT_A: case VELEXT_B:
            if (get_velocity_ext(CODEDIM, v.src == VELEXT_A ? SPINA : SPINB, it, ext.data())) return WTD_ERR_CUDA;
            src = ext.data();
            break;
        case DELTA_EXT:
            if (get_delta_ext(CODEDIM, it, (void *)(c->pots + 2 * N), ext.data())) return WTD_ERR_CUDA;
            src = ext.data();
            break;
        }
        const std::string path = s->prefix + "_" + v.name + ".wdat";
        FILE *f = fopen(path.c_str(), "ab");
        if (!f) return WTD_ERR_IO;
        const size_t n = N * (size_t)v.comps;
        size_t wrote;
        if (s->fprec) {
            std::vector<float> tmp(n);
            for (size_t p = 0; p < n; p++) tmp[p] = (float)src[p];
            wrote = fwrite(tmp.data(), sizeof(float), n, f);
        } else {
            wrote = fwrite(src, sizeof(double), n, f);
        }
        if (fclose(f) != 0 || wrote != n) return WTD_ERR_IO;
    }
    s->cycles++;
    return write_meta(s);
}

#endif
