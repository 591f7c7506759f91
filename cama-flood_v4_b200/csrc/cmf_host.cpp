// cmf_host.cpp -- host model core: the reference's initialisation chain for a stand-alone host.
//
// When the Fortran program drives the GPU it performs this initialisation itself and hands its
// module arrays to cmf_gpu_init.  This file reproduces that chain in C++ so that C++/Python
// hosts can load a case written in the reference's file formats and obtain bit-identical arrays:
//   CMF_RIVMAP_INIT   src/cmf_ctrl_maps_mod.F90:152-643  (READ_MAP_BIN, CALC_REGION, CALC_1D_SEQ,
//                                                         READ_BIFPARAM)
//   CMF_TOPO_INIT     src/cmf_ctrl_maps_mod.F90:651-1044 (READ_TOPO_BIN, SET_FLDSTG)
//   CMF_LEVEE_INIT    src/cmf_ctrl_levee_mod.F90:93-264
//   CMF_PROG_INIT     src/cmf_ctrl_vars_mod.F90:28-176   (STORAGE_SEA_SURFACE)
//   CMF_PHYSICS_FLDSTG at init, src/cmf_drv_control_mod.F90:243 (host copy of the stage scheme)
//   CMF_DAMOUT_INIT   src/cmf_ctrl_damout_mod.F90:123-308
// Arrays keep the Fortran layout and 1-based index values, so the pointers handed to the GPU
// boundary are interchangeable with the Fortran host's.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/cmf_gpu.h"

namespace {

constexpr int kImis = -9999;
inline double f32(double x) { return static_cast<double>(static_cast<float>(x)); }  // default-real literal

struct Namelist {
    bool ladpstp = true, lfplain = true, lfldout = true, lpthout = false, ldamout = false, llevee = false;
    bool lspamat = true, lkine = false, lslpmix = false, lstg_es = false, lgdwdly = false, lrosplit = false;
    bool lwevap = false, lupsinf = false, ldamh22 = false, ldamyby = false;
    double dt = 86400.0, pmanriv = 0.03, pmanfld = 0.10, pgrv = 9.8, pdstmth = 10000.0, pcadp = 0.7;
    double pminslp = f32(1.E-5), drofunit = 86400000.0;
    std::string cdiminfo = "diminfo.txt", cnextxy, cgrarea, celevtn, cnxtdst, crivlen, cfldhgt, crivwth,
                crivhgt, crivman, cpthout, clevhgt, clevfrc, cdamfile;
};

std::string upper(std::string s) {
    for (auto &c : s) c = static_cast<char>(std::toupper(static_cast<unsigned char>(c)));
    return s;
}
std::string strip(const std::string &s) {
    size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
    return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}
double fortran_real(std::string v) {
    for (auto &c : v) if (c == 'D' || c == 'd') c = 'E';
    return std::strtod(v.c_str(), nullptr);
}
bool fortran_logical(const std::string &v) {
    size_t k = v.find_first_not_of('.');
    return k != std::string::npos && (v[k] == 'T' || v[k] == 't');
}

bool read_namelist(const std::string &dir, const std::string &file, Namelist &nl) {
    std::ifstream f(dir + "/" + file);
    if (!f) return false;
    std::string line;
    while (std::getline(f, line)) {
        size_t eq = line.find('=');
        if (eq == std::string::npos) continue;
        std::string key = upper(strip(line.substr(0, eq)));
        std::string val = line.substr(eq + 1);
        size_t bang = val.find('!');
        if (bang != std::string::npos) val = val.substr(0, bang);
        val = strip(val);
        std::string sval;
        if (!val.empty() && (val[0] == '"' || val[0] == '\'')) {
            size_t e = val.find(val[0], 1);
            sval = dir + "/" + val.substr(1, e == std::string::npos ? std::string::npos : e - 1);
        }
        struct { const char *k; bool *p; } bools[] = {
            {"LADPSTP", &nl.ladpstp}, {"LFPLAIN", &nl.lfplain}, {"LFLDOUT", &nl.lfldout}, {"LPTHOUT", &nl.lpthout},
            {"LDAMOUT", &nl.ldamout}, {"LLEVEE", &nl.llevee}, {"LSPAMAT", &nl.lspamat}, {"LKINE", &nl.lkine},
            {"LSLPMIX", &nl.lslpmix}, {"LSTG_ES", &nl.lstg_es}, {"LGDWDLY", &nl.lgdwdly}, {"LROSPLIT", &nl.lrosplit},
            {"LWEVAP", &nl.lwevap}, {"LUPSINF", &nl.lupsinf}, {"LDAMH22", &nl.ldamh22}, {"LDAMYBY", &nl.ldamyby}};
        struct { const char *k; double *p; } reals[] = {
            {"DT", &nl.dt}, {"PMANRIV", &nl.pmanriv}, {"PMANFLD", &nl.pmanfld}, {"PGRV", &nl.pgrv},
            {"PDSTMTH", &nl.pdstmth}, {"PCADP", &nl.pcadp}, {"PMINSLP", &nl.pminslp}, {"DROFUNIT", &nl.drofunit}};
        struct { const char *k; std::string *p; } strs[] = {
            {"CDIMINFO", &nl.cdiminfo}, {"CNEXTXY", &nl.cnextxy}, {"CGRAREA", &nl.cgrarea}, {"CELEVTN", &nl.celevtn},
            {"CNXTDST", &nl.cnxtdst}, {"CRIVLEN", &nl.crivlen}, {"CFLDHGT", &nl.cfldhgt}, {"CRIVWTH", &nl.crivwth},
            {"CRIVHGT", &nl.crivhgt}, {"CRIVMAN", &nl.crivman}, {"CPTHOUT", &nl.cpthout}, {"CLEVHGT", &nl.clevhgt},
            {"CLEVFRC", &nl.clevfrc}, {"CDAMFILE", &nl.cdamfile}};
        for (auto &b : bools) if (key == b.k) *b.p = fortran_logical(val);
        for (auto &r : reals) if (key == r.k) *r.p = fortran_real(val);
        for (auto &s : strs) if (key == s.k) *s.p = sval;
    }
    return true;
}

template <class T>
bool read_records(const std::string &path, std::vector<T> &out, size_t n, int nrec) {
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    out.resize(n * static_cast<size_t>(nrec));
    size_t got = std::fread(out.data(), sizeof(T), out.size(), f);
    std::fclose(f);
    return got == out.size();
}

}  // namespace

struct cmf_host_model {
    Namelist nl;
    int nx = 0, ny = 0, nlfp = 0;
    int nseqmax = 0, nseqall = 0, nseqriv = 0, upnmax = 0;
    int npthout = 1, npthlev = 1, onmax = 1, inmax = 1, ndam = 0;
    std::vector<int32_t> nextx, nexty;
    std::vector<int32_t> i1seqx, i1seqy, i1next, i2vector, i1upst, i1upn, i2mask;
    std::vector<int32_t> pth_upst, pth_down, i1p_out, i1p_outn, i1p_inf, i1p_infn;
    std::vector<double> pth_dst, pth_elv, pth_wth, pth_man;
    std::vector<double> grarea, elevtn, nxtdst, rivlen, rivwth, rivhgt, fldhgt, rivman, dwnelv;
    std::vector<double> rivstomax, rivelv, fldstomax, fldgrd;
    double dfrcinc = 0.1;
    std::vector<double> levhgt, levfrc, bashgt, levdst, levbassto, levtopsto, levfilsto;
    std::vector<int32_t> damseq, damstat, i1dam;
    std::vector<double> dam_upreal, dam_qn, dam_qf, dam_qa, dam_convol, dam_fldvol, dam_emevol, dam_norvol,
        dam_adjvol, dam_r_volupa;
    // prognostics
    std::vector<double> rivsto, fldsto, rivout, fldout, rivout_pre, fldout_pre, rivdph_pre, fldsto_pre;
    std::vector<double> pthflw, pthflw_pre, damsto, daminf, levsto;
    std::string err;

    // ---- helpers ----
    size_t g(int ix, int iy) const { return static_cast<size_t>(iy - 1) * nx + (ix - 1); }
    void to_vec(const float *map, std::vector<double> &v, size_t off = 0) const {  // mapR2vecD
        for (int s = 0; s < nseqmax; s++) v[off + s] = static_cast<double>(map[g(i1seqx[s], i1seqy[s])]);
    }

    bool rivmap_init();
    bool read_bifparam();
    bool topo_init();
    bool levee_init();
    void prog_init();
    void fldstg_host();
    bool damout_init();
};

// CALC_REGION + CALC_1D_SEQ, src/cmf_ctrl_maps_mod.F90:308-525.  The ordering walks
// generation by generation: cells without upstream in row-major scan order, then every cell whose
// upstream neighbours are all placed, then the river mouths.
bool cmf_host_model::rivmap_init() {
    const size_t ng = static_cast<size_t>(nx) * ny;
    nseqmax = 0;
    for (size_t k = 0; k < ng; k++) nseqmax += (nextx[k] != kImis);
    std::vector<int32_t> nup(ng, 0), done(ng, 0);
    upnmax = 0;
    for (int iy = 1; iy <= ny; iy++)
        for (int ix = 1; ix <= nx; ix++) {
            if (nextx[g(ix, iy)] > 0) {
                int &c = nup[g(nextx[g(ix, iy)], nexty[g(ix, iy)])];
                c++;
                upnmax = std::max(upnmax, c);
            }
        }
    i1seqx.assign(nseqmax, 0);
    i1seqy.assign(nseqmax, 0);
    i2vector.assign(ng, 0);
    int n = 0;
    auto place = [&](int ix, int iy) {
        i1seqx[n] = ix;
        i1seqy[n] = iy;
        i2vector[g(ix, iy)] = ++n;
    };
    for (int iy = 1; iy <= ny; iy++)
        for (int ix = 1; ix <= nx; ix++)
            if (nextx[g(ix, iy)] > 0 && nup[g(ix, iy)] == 0) place(ix, iy);
    int lo = 0, hi = n;  // current generation [lo, hi)
    while (lo < hi) {
        for (int s = lo; s < hi; s++) {
            size_t c = g(i1seqx[s], i1seqy[s]);
            int jx = nextx[c], jy = nexty[c];
            size_t d = g(jx, jy);
            if (++done[d] == nup[d] && nextx[d] > 0) place(jx, jy);
        }
        lo = hi;
        hi = n;
    }
    nseqriv = n;
    for (int iy = 1; iy <= ny; iy++)
        for (int ix = 1; ix <= nx; ix++) {
            int v = nextx[g(ix, iy)];
            if (v < 0 && v != kImis) place(ix, iy);
        }
    nseqall = n;
    if (nseqall != nseqmax) {
        err = "river network has cells that never reach a mouth (NSEQALL /= NSEQMAX)";
        return false;
    }
    i1next.assign(nseqmax, 0);
    for (int s = 0; s < nseqall; s++) {
        size_t c = g(i1seqx[s], i1seqy[s]);
        i1next[s] = nextx[c] > 0 ? i2vector[g(nextx[c], nexty[c])] : nextx[c];
    }
    // I1UPST(NSEQMAX,UPNMAX) column-major, filled in increasing upstream order, :515-522
    const int um = std::max(upnmax, 1);
    i1upst.assign(static_cast<size_t>(nseqmax) * um, kImis);
    i1upn.assign(nseqmax, 0);
    for (int s = 0; s < nseqriv; s++) {
        int j = i1next[s] - 1;
        int k = i1upn[j]++;
        i1upst[static_cast<size_t>(k) * nseqmax + j] = s + 1;
    }
    return true;
}

// READ_BIFPARAM, src/cmf_ctrl_maps_mod.F90:531-639
bool cmf_host_model::read_bifparam() {
    std::ifstream f(nl.cpthout);
    if (!f) { err = "cannot open " + nl.cpthout; return false; }
    std::string line;
    std::getline(f, line);
    {
        std::istringstream hs(line);
        hs >> npthout >> npthlev;
    }
    const int P = npthout, Lp = npthlev;
    pth_upst.assign(P, 0); pth_down.assign(P, 0); pth_dst.assign(P, 0.0);
    pth_elv.assign(static_cast<size_t>(P) * Lp, 0.0); pth_wth.assign(static_cast<size_t>(P) * Lp, 0.0);
    pth_man.assign(Lp, 0.0);
    std::vector<int> oc(nseqmax, 0), ic(nseqmax, 0);
    for (int p = 0; p < P; p++) {
        if (!std::getline(f, line)) { err = "bifprm: fewer rows than NPTHOUT"; return false; }
        const char *s = line.c_str();
        char *e = nullptr;
        int ix = static_cast<int>(std::strtol(s, &e, 10)); s = e;
        int iy = static_cast<int>(std::strtol(s, &e, 10)); s = e;
        int jx = static_cast<int>(std::strtol(s, &e, 10)); s = e;
        int jy = static_cast<int>(std::strtol(s, &e, 10)); s = e;
        pth_dst[p] = std::strtod(s, &e); s = e;
        double pelv = std::strtod(s, &e); s = e;
        double pdph = std::strtod(s, &e); s = e;
        for (int l = 0; l < Lp; l++) { pth_wth[static_cast<size_t>(l) * P + p] = std::strtod(s, &e); s = e; }
        pth_upst[p] = i2vector[g(ix, iy)];
        pth_down[p] = i2vector[g(jx, jy)];
        if (pth_upst[p] > 0 && pth_down[p] > 0) { oc[pth_upst[p] - 1]++; ic[pth_down[p] - 1]++; }
        for (int l = 1; l <= Lp; l++) {
            double w = pth_wth[static_cast<size_t>(l - 1) * P + p];
            double &z = pth_elv[static_cast<size_t>(l - 1) * P + p];
            if (w > 0) z = (l == 1) ? pelv - pdph : (pelv + static_cast<double>(l)) - f32(2.0);
            else z = f32(1.E20);
        }
    }
    for (int l = 1; l <= Lp; l++) pth_man[l - 1] = (l == 1) ? nl.pmanriv : nl.pmanfld;
    onmax = std::max(1, *std::max_element(oc.begin(), oc.end()));
    inmax = std::max(1, *std::max_element(ic.begin(), ic.end()));
    i1p_out.assign(static_cast<size_t>(nseqmax) * onmax, 0);
    i1p_inf.assign(static_cast<size_t>(nseqmax) * inmax, 0);
    i1p_outn.assign(nseqmax, 0);
    i1p_infn.assign(nseqmax, 0);
    for (int p = 0; p < P; p++) {
        if (pth_upst[p] > 0 && pth_down[p] > 0) {
            int is = pth_upst[p] - 1, js = pth_down[p] - 1;
            i1p_out[static_cast<size_t>(i1p_outn[is]++) * nseqmax + is] = p + 1;
            i1p_inf[static_cast<size_t>(i1p_infn[js]++) * nseqmax + js] = p + 1;
        }
    }
    return true;
}

// CMF_TOPO_INIT + READ_TOPO_BIN + SET_FLDSTG, src/cmf_ctrl_maps_mod.F90:651-999
bool cmf_host_model::topo_init() {
    const size_t ng = static_cast<size_t>(nx) * ny;
    const int N = nseqmax, L = nlfp;
    std::vector<float> buf;
    struct { const std::string *path; std::vector<double> *v; } maps[] = {
        {&nl.cgrarea, &grarea}, {&nl.celevtn, &elevtn}, {&nl.cnxtdst, &nxtdst}, {&nl.crivlen, &rivlen},
        {&nl.crivhgt, &rivhgt}, {&nl.crivwth, &rivwth}, {&nl.crivman, &rivman}};
    for (auto &m : maps) {
        if (!read_records(*m.path, buf, ng, 1)) { err = "cannot read " + *m.path; return false; }
        m.v->assign(N, 0.0);
        to_vec(buf.data(), *m.v);
    }
    if (!read_records(nl.cfldhgt, buf, ng, L)) { err = "cannot read " + nl.cfldhgt; return false; }
    fldhgt.assign(static_cast<size_t>(N) * L, 0.0);
    for (int l = 0; l < L; l++) to_vec(buf.data() + static_cast<size_t>(l) * ng, fldhgt, static_cast<size_t>(l) * N);
    i2mask.assign(N, 0);
    rivstomax.assign(N, 0.0);
    rivelv.assign(N, 0.0);
    dwnelv.assign(N, 0.0);
    for (int i = 0; i < N; i++) {
        rivstomax[i] = nl.lfplain ? (rivlen[i] * rivwth[i]) * rivhgt[i] : f32(1.E18);
        rivelv[i] = elevtn[i] - rivhgt[i];
        dwnelv[i] = elevtn[i];
    }
    dfrcinc = 1.0 / static_cast<double>(L);
    fldstomax.assign(static_cast<size_t>(N) * L, 0.0);
    fldgrd.assign(static_cast<size_t>(N) * L, 0.0);
    for (int i = 0; i < N; i++) {
        double prev_sto = rivstomax[i], prev_h = 0.0;
        const double inc = (grarea[i] * (1.0 / rivlen[i])) * dfrcinc;
        for (int k = 0; k < L; k++) {
            const size_t o = static_cast<size_t>(k) * N + i;
            const double dh = fldhgt[o] - prev_h;
            fldstomax[o] = prev_sto + (rivlen[i] * (rivwth[i] + inc * (static_cast<double>(k + 1) - 0.5))) * dh;
            fldgrd[o] = dh * (1.0 / inc);
            prev_sto = fldstomax[o];
            prev_h = fldhgt[o];
        }
    }
    return true;
}

// CMF_LEVEE_INIT, src/cmf_ctrl_levee_mod.F90:93-264
bool cmf_host_model::levee_init() {
    const size_t ng = static_cast<size_t>(nx) * ny;
    const int N = nseqmax, L = nlfp;
    std::vector<float> buf;
    if (!read_records(nl.clevhgt, buf, ng, 1)) { err = "cannot read " + nl.clevhgt; return false; }
    levhgt.assign(N, 0.0);
    to_vec(buf.data(), levhgt);
    if (!read_records(nl.clevfrc, buf, ng, 1)) { err = "cannot read " + nl.clevfrc; return false; }
    levfrc.assign(N, 0.0);
    to_vec(buf.data(), levfrc);
    bashgt.assign(N, 0.0); levdst.assign(N, 0.0);
    levbassto.assign(N, 0.0); levtopsto.assign(N, 0.0); levfilsto.assign(N, 0.0);
    for (int i = 0; i < N; i++) {
        if (levhgt[i] <= 0.0 || levfrc[i] >= 1.0 || levfrc[i] < 0.0) { levhgt[i] = 0.0; levfrc[i] = 1.0; }
        levfrc[i] = std::max(0.0, std::min(1.0, levfrc[i]));
    }
    auto FSM = [&](int I, int i) -> double & { return fldstomax[static_cast<size_t>(I - 1) * N + i]; };
    auto FGR = [&](int I, int i) -> double & { return fldgrd[static_cast<size_t>(I - 1) * N + i]; };
    auto FHG = [&](int I, int i) -> double { return fldhgt[static_cast<size_t>(I - 1) * N + i]; };
    for (int i = 0; i < N; i++) {
        const double inc = (grarea[i] * (1.0 / rivlen[i])) * dfrcinc;
        // floodplain tables, recomputed identically to SET_FLDSTG
        double sto = rivstomax[i], hp = 0.0;
        for (int I = 1; I <= L; I++) {
            FSM(I, i) = sto + (rivlen[i] * (rivwth[i] + inc * (static_cast<double>(I) - 0.5))) * (FHG(I, i) - hp);
            FGR(I, i) = (FHG(I, i) - hp) * (1.0 / inc);
            sto = FSM(I, i);
            hp = FHG(I, i);
        }
        if (levhgt[i] <= 0.0) {
            bashgt[i] = levdst[i] = levbassto[i] = levtopsto[i] = levfilsto[i] = 1.E18;
            continue;
        }
        // [1] storage at the levee base and at the levee top (river side only)
        double sfil = rivstomax[i], hpre = 0.0, wfil = 0.0;
        levdst[i] = (levfrc[i] * inc) * static_cast<double>(L);
        const int ilev = static_cast<int>(levfrc[i] * static_cast<double>(L)) + 1;
        if (ilev >= 2) { sfil = FSM(ilev - 1, i); hpre = FHG(ilev - 1, i); wfil = inc * static_cast<double>(ilev - 1); }
        if (ilev <= L) {
            const double wadd = levdst[i] - wfil;
            const double hnow = wadd * FGR(ilev, i);
            bashgt[i] = hnow + hpre;
            levhgt[i] = std::max(levhgt[i], bashgt[i]);
            levbassto[i] = sfil + (((wadd * 0.5) + wfil) + rivwth[i]) * hnow * rivlen[i];
        } else {
            bashgt[i] = hpre;
            levhgt[i] = std::max(levhgt[i], bashgt[i]);
            levbassto[i] = sfil;
        }
        levtopsto[i] = levbassto[i] + ((levdst[i] + rivwth[i]) * (levhgt[i] - bashgt[i])) * rivlen[i];
        // [2] storage when both sides are filled to the levee crown
        int I = 1;
        sfil = rivstomax[i];
        wfil = rivwth[i];
        hpre = 0.0;
        while (I <= L && levhgt[i] > FHG(I, i)) {
            sfil = FSM(I, i);
            wfil = wfil + inc;
            hpre = FHG(I, i);
            I++;
        }
        const double hnow = levhgt[i] - hpre;
        if (I <= L) {
            const double wadd = hnow / FGR(I, i);
            levfilsto[i] = sfil + ((wadd * 0.5) + wfil) * hnow * rivlen[i];
        } else {
            levfilsto[i] = sfil + (wfil * hnow) * rivlen[i];
        }
    }
    return true;
}

// CMF_PROG_INIT: zero state and STORAGE_SEA_SURFACE, src/cmf_ctrl_vars_mod.F90:129-176
void cmf_host_model::prog_init() {
    const int N = nseqmax;
    const size_t PL = static_cast<size_t>(npthout) * npthlev;
    for (auto *v : {&rivsto, &fldsto, &rivout, &fldout, &rivout_pre, &fldout_pre, &rivdph_pre, &fldsto_pre,
                    &damsto, &daminf, &levsto})
        v->assign(N, 0.0);
    pthflw.assign(PL, 0.0);
    pthflw_pre.assign(PL, 0.0);
    auto fill = [&](int i, double sea) {
        double d = std::min(std::max(sea - rivelv[i], 0.0), rivhgt[i]);
        rivsto[i] = std::min((d * rivlen[i]) * rivwth[i], rivstomax[i] * 1.0);
        rivdph_pre[i] = d;
    };
    for (int i = nseqriv; i < nseqall; i++) fill(i, dwnelv[i]);
    for (int i = nseqriv - 1; i >= 0; i--) {
        const int j = i1next[i] - 1;
        fill(i, rivelv[j] + rivdph_pre[j]);
    }
}

// The only state-changing effect of the init-time CMF_PHYSICS_FLDSTG (src/cmf_drv_control_mod.F90:243)
// is the river/floodplain split of the storage (and P2LEVSTO with levees); CMF_DAMOUT_INIT then reads
// P2RIVSTO+P2FLDSTO.  STORAGE_SEA_SURFACE never exceeds the bank, so the split leaves every cell
// in-bank and unchanged; with levees the protected-side storage stays zero for the same reason.
void cmf_host_model::fldstg_host() {}

// CMF_DAMOUT_INIT, src/cmf_ctrl_damout_mod.F90:123-308 (no restart)
bool cmf_host_model::damout_init() {
    std::ifstream f(nl.cdamfile);
    if (!f) { err = "cannot open " + nl.cdamfile; return false; }
    std::string line;
    std::getline(f, line);
    ndam = std::atoi(line.c_str());
    std::getline(f, line);  // header
    damseq.assign(ndam, kImis); damstat.assign(ndam, kImis); i1dam.assign(nseqmax, 0);
    for (auto *v : {&dam_upreal, &dam_qn, &dam_qf, &dam_qa, &dam_convol, &dam_fldvol, &dam_emevol, &dam_norvol,
                    &dam_adjvol, &dam_r_volupa})
        v->assign(ndam, 0.0);
    int placed = 0;
    for (int d = 0; d < ndam; d++) {
        if (!std::getline(f, line)) { err = "dam table shorter than NDAM"; return false; }
        for (auto &c : line) if (c == ',') c = ' ';
        std::istringstream rs(line);
        std::string id, name, lat, lon, upa, six, siy, sfld, scon, stot, sqn, sqf;
        rs >> id >> name >> lat >> lon >> upa >> six >> siy >> sfld >> scon >> stot >> sqn >> sqf;
        if (sqf.empty()) { err = "malformed dam row"; return false; }
        dam_upreal[d] = std::strtod(upa.c_str(), nullptr);
        const int ix = std::atoi(six.c_str()), iy = std::atoi(siy.c_str());
        dam_qn[d] = std::strtod(sqn.c_str(), nullptr);
        dam_qf[d] = std::strtod(sqf.c_str(), nullptr);
        dam_fldvol[d] = std::strtod(sfld.c_str(), nullptr) * 1.E6;
        dam_convol[d] = std::strtod(scon.c_str(), nullptr) * 1.E6;
        dam_emevol[d] = dam_convol[d] + dam_fldvol[d] * 0.95;
        if (ix <= 0 || ix > nx || iy <= 0 || iy > ny) continue;
        const int s = i2vector[g(ix, iy)];
        if (s <= 0 || i1next[s - 1] == kImis) continue;
        placed++;
        damseq[d] = s;
        damstat[d] = 2;
        i1dam[s - 1] = 1;
        i2mask[s - 1] = 2;
        if (nl.ldamh22) {
            dam_norvol[d] = dam_convol[d] * 0.5;
            dam_r_volupa[ndam - 1] = (dam_fldvol[d] * f32(1.E-6)) / dam_upreal[d];  // index NDAM, as the reference writes it
        } else {
            const double vyr = dam_qn[d] * 31536000.0;                         // 365.*24.*60.*60. (exact in FP32)
            const double qsto = ((dam_convol[d] * f32(0.7)) + vyr / 4.0) / 15552000.0;  // 180.*24.*60.*60.
            dam_qn[d] = std::min(dam_qn[d], qsto) * 1.5;
            dam_adjvol[d] = dam_convol[d] + dam_fldvol[d] * f32(0.1);
            dam_qa[d] = (dam_qn[d] + dam_qf[d]) * 0.5;
        }
    }
    if (placed == 0) { err = "none of the given dams is inside the domain"; return false; }
    for (int i = 0; i < nseqall; i++) {
        const int j = i1next[i] - 1;
        if (i1dam[i] <= 0 && i1next[i] > 0 && (i1dam[j] == 1 || i1dam[j] == 11)) { i1dam[i] = 10; i2mask[i] = 1; }
        if (i1dam[i] == 1 && i1next[i] > 0 && (i1dam[j] == 1 || i1dam[j] == 11)) { i1dam[i] = 11; i2mask[i] = 2; }
    }
    for (int d = 0; d < ndam; d++) {
        if (damstat[d] == kImis) continue;
        const int s = damseq[d] - 1;
        damsto[s] = rivsto[s] + fldsto[s];
        if (damstat[d] != -1 && damsto[s] < dam_convol[d]) {
            damsto[s] = dam_convol[d];
            rivsto[s] = dam_convol[d];
            fldsto[s] = 0.0;
        }
    }
    if (nl.lpthout) {
        for (int p = 0; p < npthout; p++) {
            const int u = pth_upst[p], v = pth_down[p];
            if (u <= 0 || v <= 0) continue;
            if (i1dam[u - 1] > 0 || i1dam[v - 1] > 0)
                for (int l = 0; l < npthlev; l++) pth_elv[static_cast<size_t>(l) * npthout + p] = f32(1.E20);
        }
    }
    return true;
}

extern "C" {

int cmf_host_load(const char *casedir, const char *nmlfile, cmf_host_model **out) {
    if (!casedir || !out) return CMF_E_ARG;
    *out = nullptr;
    auto *hm = new cmf_host_model();
    const std::string dir(casedir);
    const std::string nml = nmlfile ? nmlfile : "input_cmf.nam";
    auto fail = [&](const std::string &why) {
        std::fprintf(stderr, "cmf_host_load: %s\n", why.c_str());
        delete hm;
        return CMF_E_IO;
    };
    if (!read_namelist(dir, nml, hm->nl)) return fail("cannot read namelist " + dir + "/" + nml);
    {
        std::ifstream f(hm->nl.cdiminfo.find('/') == std::string::npos ? dir + "/" + hm->nl.cdiminfo : hm->nl.cdiminfo);
        std::ifstream f2(dir + "/diminfo.txt");
        std::ifstream &src = f ? f : f2;
        if (!src) return fail("cannot read diminfo");
        std::string l1, l2, l3;
        std::getline(src, l1); std::getline(src, l2); std::getline(src, l3);
        hm->nx = std::atoi(l1.c_str()); hm->ny = std::atoi(l2.c_str()); hm->nlfp = std::atoi(l3.c_str());
    }
    const size_t ng = static_cast<size_t>(hm->nx) * hm->ny;
    std::vector<int32_t> nxy;
    if (!read_records(hm->nl.cnextxy, nxy, ng, 2)) return fail("cannot read " + hm->nl.cnextxy);
    hm->nextx.assign(nxy.begin(), nxy.begin() + ng);
    hm->nexty.assign(nxy.begin() + ng, nxy.end());
    if (!hm->rivmap_init()) return fail(hm->err);
    if (hm->nl.lpthout) {
        if (!hm->read_bifparam()) return fail(hm->err);
    } else {
        hm->npthout = 1; hm->npthlev = 1; hm->onmax = 1; hm->inmax = 1;
        hm->pth_upst.assign(1, 0); hm->pth_down.assign(1, 0); hm->pth_dst.assign(1, 0.0);
        hm->pth_elv.assign(1, 0.0); hm->pth_wth.assign(1, 0.0); hm->pth_man.assign(1, 0.0);
        hm->i1p_out.assign(hm->nseqmax, 0); hm->i1p_inf.assign(hm->nseqmax, 0);
        hm->i1p_outn.assign(hm->nseqmax, 0); hm->i1p_infn.assign(hm->nseqmax, 0);
    }
    if (!hm->topo_init()) return fail(hm->err);
    if (hm->nl.llevee && !hm->levee_init()) return fail(hm->err);
    hm->prog_init();
    hm->fldstg_host();
    if (hm->nl.ldamout) {
        if (!hm->damout_init()) return fail(hm->err);
    } else {
        hm->i1dam.assign(hm->nseqmax, 0);
    }
    *out = hm;
    return CMF_OK;
}

void cmf_host_free(cmf_host_model *hm) { delete hm; }

int cmf_host_describe(const cmf_host_model *hm, cmf_dims *dims, cmf_params *params, cmf_map_ptrs *maps,
                      cmf_opts *opts, double *dt) {
    if (!hm) return CMF_E_ARG;
    auto &n = hm->nl;
    if (dims) {
        *dims = cmf_dims{};
        dims->nseqall = hm->nseqall; dims->nseqriv = hm->nseqriv; dims->nseqmax = hm->nseqmax;
        dims->nlfp = hm->nlfp; dims->upnmax = std::max(hm->upnmax, 1); dims->npthout = hm->npthout;
        dims->npthlev = hm->npthlev; dims->onmax = hm->onmax; dims->inmax = hm->inmax;
        dims->ndam = n.ldamout ? hm->ndam : 0; dims->nmembers = 1;
    }
    if (params) {
        params->pgrv = n.pgrv; params->pmanfld = n.pmanfld; params->pdstmth = n.pdstmth;
        params->pcadp = n.pcadp; params->pminslp = n.pminslp; params->dfrcinc = hm->dfrcinc;
    }
    if (maps) {
        *maps = cmf_map_ptrs{};
        maps->i1next = hm->i1next.data(); maps->i1upst = hm->i1upst.data(); maps->i1upn = hm->i1upn.data();
        maps->i2mask = hm->i2mask.data();
        maps->rivelv = hm->rivelv.data(); maps->elevtn = hm->elevtn.data(); maps->nxtdst = hm->nxtdst.data();
        maps->rivwth = hm->rivwth.data(); maps->rivhgt = hm->rivhgt.data(); maps->rivlen = hm->rivlen.data();
        maps->rivman = hm->rivman.data(); maps->grarea = hm->grarea.data(); maps->rivstomax = hm->rivstomax.data();
        maps->dwnelv = hm->dwnelv.data(); maps->fldstomax = hm->fldstomax.data(); maps->fldgrd = hm->fldgrd.data();
        maps->fldhgt = hm->fldhgt.data();
        maps->pth_upst = hm->pth_upst.data(); maps->pth_down = hm->pth_down.data(); maps->pth_dst = hm->pth_dst.data();
        maps->pth_elv = hm->pth_elv.data(); maps->pth_wth = hm->pth_wth.data(); maps->pth_man = hm->pth_man.data();
        maps->i1p_out = hm->i1p_out.data(); maps->i1p_outn = hm->i1p_outn.data();
        maps->i1p_inf = hm->i1p_inf.data(); maps->i1p_infn = hm->i1p_infn.data();
        if (n.llevee) {
            maps->levhgt = hm->levhgt.data(); maps->levfrc = hm->levfrc.data(); maps->bashgt = hm->bashgt.data();
            maps->levdst = hm->levdst.data(); maps->levbassto = hm->levbassto.data();
            maps->levtopsto = hm->levtopsto.data(); maps->levfilsto = hm->levfilsto.data();
        }
        if (n.ldamout) {
            maps->damseq = hm->damseq.data(); maps->damstat = hm->damstat.data(); maps->i1dam = hm->i1dam.data();
            maps->dam_qn = hm->dam_qn.data(); maps->dam_qf = hm->dam_qf.data(); maps->dam_qa = hm->dam_qa.data();
            maps->dam_convol = hm->dam_convol.data(); maps->dam_fldvol = hm->dam_fldvol.data();
            maps->dam_emevol = hm->dam_emevol.data(); maps->dam_norvol = hm->dam_norvol.data();
            maps->dam_adjvol = hm->dam_adjvol.data(); maps->dam_r_volupa = hm->dam_r_volupa.data();
        }
    }
    if (opts) {
        *opts = cmf_opts{};
        opts->ladpstp = n.ladpstp; opts->lfldout = n.lfldout; opts->lpthout = n.lpthout; opts->ldamout = n.ldamout;
        opts->llevee = n.llevee; opts->lspamat = n.lspamat; opts->lkine = n.lkine; opts->lslpmix = n.lslpmix;
        opts->lstg_es = n.lstg_es; opts->lgdwdly = n.lgdwdly; opts->lrosplit = n.lrosplit; opts->lwevap = n.lwevap;
        opts->lupsinf = n.lupsinf; opts->ldamh22 = n.ldamh22; opts->ldamyby = n.ldamyby;
        opts->ldiag = 1; opts->launch_mode = 0; opts->device = 0; opts->block_size = 0; opts->ldiag_output = 0;
    }
    if (dt) *dt = n.dt;
    return CMF_OK;
}

int cmf_host_state(cmf_host_model *hm, cmf_state_ptrs *st) {
    if (!hm || !st) return CMF_E_ARG;
    st->rivsto = hm->rivsto.data(); st->fldsto = hm->fldsto.data();
    st->rivout = hm->rivout.data(); st->fldout = hm->fldout.data();
    st->rivout_pre = hm->rivout_pre.data(); st->fldout_pre = hm->fldout_pre.data();
    st->rivdph_pre = hm->rivdph_pre.data(); st->fldsto_pre = hm->fldsto_pre.data();
    st->pthflw = hm->pthflw.data(); st->pthflw_pre = hm->pthflw_pre.data();
    st->damsto = hm->damsto.data(); st->daminf = hm->daminf.data(); st->levsto = hm->levsto.data();
    return CMF_OK;
}

int cmf_host_conv_resol(const cmf_host_model *hm, const double *map, double *out) {
    if (!hm || !map || !out) return CMF_E_ARG;
    const double rmis = f32(1.E20);
    for (int i = 0; i < hm->nseqmax; i++) {
        const double v = map[hm->g(hm->i1seqx[i], hm->i1seqy[i])];
        out[i] = (v != rmis) ? std::max((v * hm->grarea[i]) / hm->nl.drofunit, 0.0) : 0.0;
    }
    return CMF_OK;
}

// ---- binary restart (CMF_RESTART_WRITE / CMF_RESTART_INIT, src/cmf_ctrl_restart_mod.F90:91-482) ----
// Record layout: one NX x NY map per variable (FP64 when LRESTDBL, else FP32), cells outside the
// sequence filled with DMIS / RMIS = 1.E20, in the order rivsto, fldsto, [rivout_pre, fldout_pre,
// rivdph_pre, fldsto_pre unless LSTOONLY], [damsto if LDAMOUT], [levsto if LLEVEE]; bifurcation
// flows D1PTHFLW_PRE as one (NPTHOUT,NPTHLEV) record in <file>.pth.
namespace {
int rest_put(const cmf_host_model *hm, FILE *f, const double *vec, bool dbl) {
    const size_t nxy = static_cast<size_t>(hm->nx) * hm->ny;
    size_t w;
    if (dbl) {
        std::vector<double> map(nxy, 1.E20);
        for (int i = 0; i < hm->nseqmax; i++) map[hm->g(hm->i1seqx[i], hm->i1seqy[i])] = vec[i];
        w = std::fwrite(map.data(), sizeof(double), nxy, f);
    } else {
        std::vector<float> map(nxy, 1.E20f);
        for (int i = 0; i < hm->nseqmax; i++) map[hm->g(hm->i1seqx[i], hm->i1seqy[i])] = static_cast<float>(vec[i]);
        w = std::fwrite(map.data(), sizeof(float), nxy, f);
    }
    return w == nxy ? CMF_OK : CMF_E_IO;
}
int rest_get(const cmf_host_model *hm, FILE *f, double *vec, bool dbl) {
    const size_t nxy = static_cast<size_t>(hm->nx) * hm->ny;
    std::vector<double> map(nxy);
    if (dbl) {
        if (std::fread(map.data(), sizeof(double), nxy, f) != nxy) return CMF_E_IO;
    } else {
        std::vector<float> r(nxy);
        if (std::fread(r.data(), sizeof(float), nxy, f) != nxy) return CMF_E_IO;
        for (size_t k = 0; k < nxy; k++) map[k] = static_cast<double>(r[k]);
    }
    for (int i = 0; i < hm->nseqmax; i++) vec[i] = map[hm->g(hm->i1seqx[i], hm->i1seqy[i])];
    return CMF_OK;
}
}  // namespace

int cmf_host_write_restart(const cmf_host_model *hm, const cmf_state_ptrs *st, const char *file, int32_t lrestdbl,
                           int32_t lstoonly) {
    if (!hm || !st || !file || !st->rivsto || !st->fldsto) return CMF_E_ARG;
    const auto &n = hm->nl;
    if (!lstoonly && (!st->rivout_pre || !st->fldout_pre || !st->rivdph_pre || !st->fldsto_pre)) return CMF_E_ARG;
    if ((n.ldamout && !st->damsto) || (n.llevee && !st->levsto) || (n.lpthout && !st->pthflw_pre)) return CMF_E_ARG;
    FILE *f = std::fopen(file, "wb");
    if (!f) return CMF_E_IO;
    const bool dbl = lrestdbl != 0;
    int rc = rest_put(hm, f, st->rivsto, dbl);
    if (!rc) rc = rest_put(hm, f, st->fldsto, dbl);
    if (!rc && !lstoonly) {
        for (const double *v : {st->rivout_pre, st->fldout_pre, st->rivdph_pre, st->fldsto_pre})
            if (!rc) rc = rest_put(hm, f, v, dbl);
    }
    if (!rc && n.ldamout) rc = rest_put(hm, f, st->damsto, dbl);
    if (!rc && n.llevee) rc = rest_put(hm, f, st->levsto, dbl);
    if (std::fclose(f) != 0 && !rc) rc = CMF_E_IO;
    if (rc || !n.lpthout) return rc;
    const std::string pth = std::string(file) + ".pth";
    FILE *g = std::fopen(pth.c_str(), "wb");
    if (!g) return CMF_E_IO;
    const size_t np = static_cast<size_t>(hm->npthout) * hm->npthlev;
    size_t w;
    if (dbl) {
        w = std::fwrite(st->pthflw_pre, sizeof(double), np, g);
    } else {
        std::vector<float> r(np);
        for (size_t k = 0; k < np; k++) r[k] = static_cast<float>(st->pthflw_pre[k]);
        w = std::fwrite(r.data(), sizeof(float), np, g);
    }
    if (std::fclose(g) != 0 || w != np) return CMF_E_IO;
    return CMF_OK;
}

int cmf_host_read_restart(const cmf_host_model *hm, const cmf_state_ptrs *st, const char *file, int32_t lrestdbl,
                          int32_t lstoonly) {
    if (!hm || !st || !file || !st->rivsto || !st->fldsto || !st->rivout || !st->fldout || !st->rivout_pre ||
        !st->fldout_pre || !st->rivdph_pre || !st->fldsto_pre)
        return CMF_E_ARG;
    const auto &n = hm->nl;
    if ((n.ldamout && !st->damsto) || (n.llevee && !st->levsto) || (n.lpthout && (!st->pthflw_pre || !st->pthflw)))
        return CMF_E_ARG;
    const size_t N = static_cast<size_t>(hm->nseqmax), np = static_cast<size_t>(hm->npthout) * hm->npthlev;
    for (double *v : {st->rivsto, st->fldsto, st->rivout, st->fldout, st->rivout_pre, st->fldout_pre, st->rivdph_pre,
                      st->fldsto_pre})
        std::fill(v, v + N, 0.0);
    if (n.ldamout) std::fill(st->damsto, st->damsto + N, 0.0);
    if (n.llevee) std::fill(st->levsto, st->levsto + N, 0.0);
    if (n.lpthout) { std::fill(st->pthflw, st->pthflw + np, 0.0); std::fill(st->pthflw_pre, st->pthflw_pre + np, 0.0); }
    FILE *f = std::fopen(file, "rb");
    if (!f) return CMF_E_IO;
    const bool dbl = lrestdbl != 0;
    int rc = rest_get(hm, f, st->rivsto, dbl);
    if (!rc) rc = rest_get(hm, f, st->fldsto, dbl);
    if (!rc && !lstoonly) {
        for (double *v : {st->rivout_pre, st->fldout_pre, st->rivdph_pre, st->fldsto_pre})
            if (!rc) rc = rest_get(hm, f, v, dbl);
    }
    if (!rc && n.ldamout) rc = rest_get(hm, f, st->damsto, dbl);
    if (!rc && n.llevee) rc = rest_get(hm, f, st->levsto, dbl);
    std::fclose(f);
    if (rc) return rc;
    if (n.lpthout && !lstoonly) {
        const std::string pth = std::string(file) + ".pth";
        FILE *g = std::fopen(pth.c_str(), "rb");
        if (!g) return CMF_E_IO;
        size_t r;
        if (dbl) {
            r = std::fread(st->pthflw_pre, sizeof(double), np, g);
        } else {
            std::vector<float> v(np);
            r = std::fread(v.data(), sizeof(float), np, g);
            for (size_t k = 0; k < np; k++) st->pthflw_pre[k] = static_cast<double>(v[k]);
        }
        std::fclose(g);
        if (r != np) return CMF_E_IO;
    }
    if (lstoonly) std::copy(st->fldsto, st->fldsto + N, st->fldsto_pre);   // :130-132
    return CMF_OK;
}

int cmf_host_read_inpmat(const cmf_host_model *hm, const char *file, int32_t inpn, int32_t *inpx, int32_t *inpy,
                         double *inpa) {
    if (!hm || !file || inpn < 1 || !inpx || !inpy || !inpa) return CMF_E_ARG;
    FILE *f = std::fopen(file, "rb");
    if (!f) return CMF_E_IO;
    const size_t nxy = static_cast<size_t>(hm->nx) * hm->ny, N = static_cast<size_t>(hm->nseqmax);
    std::vector<int32_t> ib(nxy);
    std::vector<float> rb(nxy);
    int rc = CMF_OK;
    // records 1..INPN: INPX, INPN+1..2*INPN: INPY, 2*INPN+1..3*INPN: INPA (direct access, RECL = 4*NX*NY)
    for (int part = 0; part < 3 && !rc; part++) {
        for (int k = 0; k < inpn && !rc; k++) {
            const size_t got = part < 2 ? std::fread(ib.data(), 4, nxy, f) : std::fread(rb.data(), 4, nxy, f);
            if (got != nxy) { rc = CMF_E_IO; break; }
            for (size_t i = 0; i < N; i++) {
                const size_t gi = hm->g(hm->i1seqx[i], hm->i1seqy[i]);
                if (part == 0) inpx[k * N + i] = ib[gi];                            // mapI2vecI
                else if (part == 1) inpy[k * N + i] = ib[gi];
                else inpa[k * N + i] = static_cast<double>(rb[gi]);              // mapR2vecD
            }
        }
    }
    std::fclose(f);
    return rc;
}

double cmf_host_drofunit(const cmf_host_model *hm) { return hm ? hm->nl.drofunit : 0.0; }

int cmf_host_map_to_vec(const cmf_host_model *hm, const float *map, double *vec) {
    if (!hm || !map || !vec) return CMF_E_ARG;
    for (int i = 0; i < hm->nseqmax; i++) vec[i] = static_cast<double>(map[hm->g(hm->i1seqx[i], hm->i1seqy[i])]);
    return CMF_OK;
}

int cmf_host_grid(const cmf_host_model *hm, int32_t *nx, int32_t *ny, int32_t *sx, int32_t *sy) {
    if (!hm) return CMF_E_ARG;
    if (nx) *nx = hm->nx;
    if (ny) *ny = hm->ny;
    if (sx) std::copy(hm->i1seqx.begin(), hm->i1seqx.end(), sx);
    if (sy) std::copy(hm->i1seqy.begin(), hm->i1seqy.end(), sy);
    return CMF_OK;
}

}  // extern "C"
