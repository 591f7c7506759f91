/*
 * cmf_oracle.c -- CPU FP64 restatement of CaMa-Flood v4's physics time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the correctness oracle for the B200 path and the
 * timed CPU baseline.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline and
 * reference arms may load it, and only as the checker.  The product never links it.
 *
 * PARITY UNPINNED: the reference is Fortran 90 and no Fortran compiler exists on this machine
 * or the GPU box, and the reference ships no golden vectors or known-answer tests for this path.
 * This restatement follows the cited Fortran statement by statement (same loop order, same
 * left-to-right evaluation order, same single-precision literal promotions) and is checked
 * against hand-derived known-answer tests and the reference's own water-budget identities.
 *
 * Build: gcc -O2 -ffp-contract=off -fno-fast-math (glibc pow/sqrt), optionally -fopenmp for the
 * timed baseline; OpenMP pragmas sit only on loops the reference parallelises without atomics.
 *
 * Fortran -> C conventions used throughout:
 *   - sequence index ISEQ (1-based) is i = ISEQ-1; I1NEXT keeps mouth codes (negative) and stores
 *     river links 0-based, so "I1NEXT(ISEQ)>0" becomes "i1next[i] >= 0";
 *   - (NSEQMAX,1,NLFP) arrays are layer-major [I][i]; (NPTHOUT,NPTHLEV) arrays are [ILEV][IPTH];
 *   - x**(-1.) -> 1.0/x, x**2._JPRB -> x*x, x**1.0 -> x (what gfortran emits), every other
 *     non-integral power is glibc pow();
 *   - a default-real literal (no _JPRB) is the float value promoted to double: F(1.E-5).
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <ctype.h>
#ifdef _OPENMP
#include <omp.h>
#define OMP_FOR _Pragma("omp parallel for schedule(static)")
#else
#define OMP_FOR
#endif

#define F(x) ((double)(float)(x))   /* default-real literal promoted to JPRB */
#define IMIS (-9999)

static inline double dmax(double a, double b) { return (a > b) ? a : b; }

/* Sensitivity probe (tests only): when orc_pow_perturb is non-zero, every pow() result whose
 * low mantissa bit pattern matches a hash is moved by one ulp.  Used to measure how far the
 * reference algorithm itself amplifies last-bit differences of the math library. */
static unsigned orc_pow_perturb = 0;
void orc_set_pow_perturb(unsigned v) { orc_pow_perturb = v; }
static inline double opow(double x, double y) {
    double r = pow(x, y);
    if (orc_pow_perturb) {
        uint64_t b; memcpy(&b, &r, 8);
        if (((b * 0x9E3779B97F4A7C15ull) >> 61) < orc_pow_perturb) r = nextafter(r, (b & 1) ? 0.0 : 1e308);
    }
    return r;
}
static inline double dmin(double a, double b) { return (a < b) ? a : b; }

typedef struct {
    /* ---- dimensions (src/yos_cmf_input.F90, src/yos_cmf_map.F90) */
    int nx, ny, nlfp, nseqmax, nseqall, nseqriv, npthout, npthlev, ndam, upnmax, onmax, inmax;
    /* ---- options (src/cmf_ctrl_nmlist_mod.F90:77-115) */
    int ladpstp, lfplain, lfldout, lpthout, ldamout, llevee, lspamat, lstg_es;
    int ldamh22, ldamyby, livnorm, lmeansl;
    double dt, pmanriv, pmanfld, pgrv, pdstmth, pcadp, pminslp, dfrcinc, drofunit;
    char cnextxy[512], cgrarea[512], celevtn[512], cnxtdst[512], crivlen[512], cfldhgt[512];
    char crivwth[512], crivhgt[512], crivman[512], cpthout[512], clevhgt[512], clevfrc[512], cdamfile[512];
    /* ---- network (CALC_1D_SEQ, READ_BIFPARAM) */
    int *nextx, *nexty, *i1seqx, *i1seqy, *i1next, *i2vector, *i1upst, *i1upn;
    int *i1p_out, *i1p_outn, *i1p_inf, *i1p_infn;
    int *pth_upst, *pth_down;
    double *pth_dst, *pth_elv, *pth_wth, *pth_man;
    /* ---- topography (CMF_TOPO_INIT) */
    double *grarea, *elevtn, *nxtdst, *rivlen, *rivwth, *rivhgt, *fldhgt, *rivman, *dwnelv;
    double *rivstomax, *rivelv, *fldstomax, *fldgrd;
    int *i2mask;
    /* ---- levee (CMF_LEVEE_INIT) */
    double *levhgt, *levfrc, *bashgt, *levdst, *levbassto, *levtopsto, *levfilsto;
    /* ---- dam (CMF_DAMOUT_INIT) */
    int *damseq, *damstat, *i1dam;
    double *upreal, *r_volupa, *qf, *qn, *emevol, *fldvol, *convol, *norvol, *adjvol, *qa;
    /* ---- prognostics (src/yos_cmf_prog.F90) */
    double *runoff, *rofsub, *rivsto, *fldsto, *rivout, *fldout, *rivout_pre, *fldout_pre;
    double *rivdph_pre, *fldsto_pre, *pthflw, *pthflw_pre, *gdwrtn, *damsto, *daminf, *levsto;
    /* ---- diagnostics (src/yos_cmf_diag.F90) */
    double *rivinf, *rivdph, *rivvel, *fldinf, *flddph, *fldfrc, *fldare, *pthout, *pthinf;
    double *sfcelv, *outflw, *storge, *levdph, *pthflwsum, *stoout, *p_rivinf, *p_fldinf, *p_pthout;
    double *rate, *sfcelv_pre, *dwnelv_pre, *flddph_pre, *sfcelv_lev;
    /* ---- sub-step averages (src/cmf_calc_diag_mod.F90) */
    double nadd_adp;
    double *rivout_a, *fldout_a, *outflw_a, *rivvel_a, *pthout_a, *gdwrtn_a, *runoff_a, *rofsub_a;
    double *daminf_a, *storge_m, *outflw_m, *rivdph_m, *pthflw_a, *pthflwsum_a;
    /* ---- output-interval averages (src/yos_cmf_diag.F90:82-103) */
    double nadd_out;
    double *rivout_o, *fldout_o, *outflw_o, *rivvel_o, *pthout_o, *gdwrtn_o, *runoff_o, *rofsub_o, *daminf_o;
    double *storge_om, *outflw_om, *rivdph_om, *pthflw_o;
    /* ---- budgets (src/yos_cmf_diag.F90 P0GLB*) */
    double glbstopre, glbstonxt, glbstonew, glbrivinf, glbrivout;
    double glbstopre2, glbstonew2, glbrivsto, glbfldsto, glblevsto, glbfldare;
    double dam_miss;
    int last_nt;
    double last_dt, last_dtmin;
    void (*substep_hook)(void *ctx, int it);   /* tests only: sees each sub-step's fields */
    void *substep_ctx;
    char err[256];
} orc_model;

/* ============================================================================ namelist */
static void trim(char *s) {
    char *p = s; while (*p && isspace((unsigned char)*p)) p++;
    if (p != s) memmove(s, p, strlen(p) + 1);
    size_t n = strlen(s); while (n && isspace((unsigned char)s[n - 1])) s[--n] = 0;
}
static double nml_real(const char *v) {
    char buf[128]; size_t k = 0;
    for (; *v && k < sizeof(buf) - 1; v++) buf[k++] = (*v == 'D' || *v == 'd') ? 'E' : *v;
    buf[k] = 0; return strtod(buf, NULL);
}
static int nml_logical(const char *v) {
    while (*v == '.') v++; return (*v == 'T' || *v == 't');
}
static int read_namelist(orc_model *m, const char *dir, const char *file) {
    char path[1024]; snprintf(path, sizeof path, "%s/%s", dir, file);
    FILE *f = fopen(path, "r");
    if (!f) { snprintf(m->err, sizeof m->err, "cannot open %s", path); return -1; }
    char line[1024];
    while (fgets(line, sizeof line, f)) {
        char *eq = strchr(line, '='); if (!eq) continue;
        *eq = 0; char key[128]; strncpy(key, line, 127); key[127] = 0; trim(key);
        char val[900]; strncpy(val, eq + 1, 899); val[899] = 0;
        char *bang = strchr(val, '!'); if (bang) *bang = 0; trim(val);
        for (char *p = key; *p; p++) *p = (char)toupper((unsigned char)*p);
        char sval[900] = {0};
        if (val[0] == '"' || val[0] == '\'') { char q = val[0]; char *e = strchr(val + 1, q); if (e) *e = 0; snprintf(sval, sizeof sval, "%s/%s", dir, val + 1); }
#define L(K, V) if (!strcmp(key, K)) { m->V = nml_logical(val); continue; }
#define R(K, V) if (!strcmp(key, K)) { m->V = nml_real(val); continue; }
#define S(K, V) if (!strcmp(key, K)) { snprintf(m->V, sizeof m->V, "%s", sval); continue; }
        L("LADPSTP", ladpstp) L("LFPLAIN", lfplain) L("LFLDOUT", lfldout) L("LPTHOUT", lpthout)
        L("LDAMOUT", ldamout) L("LLEVEE", llevee) L("LSPAMAT", lspamat) L("LSTG_ES", lstg_es)
        L("LDAMH22", ldamh22) L("LDAMYBY", ldamyby) L("LIVNORM", livnorm) L("LMEANSL", lmeansl)
        R("DT", dt) R("PMANRIV", pmanriv) R("PMANFLD", pmanfld) R("PGRV", pgrv) R("PDSTMTH", pdstmth)
        R("PCADP", pcadp) R("PMINSLP", pminslp) R("DROFUNIT", drofunit)
        S("CNEXTXY", cnextxy) S("CGRAREA", cgrarea) S("CELEVTN", celevtn) S("CNXTDST", cnxtdst)
        S("CRIVLEN", crivlen) S("CFLDHGT", cfldhgt) S("CRIVWTH", crivwth) S("CRIVHGT", crivhgt)
        S("CRIVMAN", crivman) S("CPTHOUT", cpthout) S("CLEVHGT", clevhgt) S("CLEVFRC", clevfrc)
        S("CDAMFILE", cdamfile)
#undef L
#undef R
#undef S
    }
    fclose(f);
    return 0;
}

/* ============================================================================ file readers */
static int read_f32_records(const char *path, float *out, size_t n, int nrec) {
    FILE *f = fopen(path, "rb"); if (!f) return -1;
    size_t got = fread(out, sizeof(float), n * (size_t)nrec, f); fclose(f);
    return got == n * (size_t)nrec ? 0 : -2;
}
static int read_i32_records(const char *path, int *out, size_t n, int nrec) {
    FILE *f = fopen(path, "rb"); if (!f) return -1;
    size_t got = fread(out, sizeof(int), n * (size_t)nrec, f); fclose(f);
    return got == n * (size_t)nrec ? 0 : -2;
}
static double *dalloc(size_t n) { return (double *)calloc(n ? n : 1, sizeof(double)); }
static int *ialloc(size_t n) { return (int *)calloc(n ? n : 1, sizeof(int)); }

/* mapR2vecD: src/cmf_utils_mod.F90:282-303 (FP32 map -> FP64 vector in sequence order) */
static void map_r2vec(const orc_model *m, const float *map, double *vec) {
    for (int i = 0; i < m->nseqmax; i++) {
        int ix = m->i1seqx[i], iy = m->i1seqy[i];
        vec[i] = (double)map[(size_t)(iy - 1) * m->nx + (ix - 1)];
    }
}

/* ============================================================================ CALC_1D_SEQ */
/* src/cmf_ctrl_maps_mod.F90:403-525 (serial by design) */
static int calc_1d_seq(orc_model *m) {
    int nx = m->nx, ny = m->ny;
    size_t ng = (size_t)nx * ny;
    int *nupst = ialloc(ng), *upnow = ialloc(ng);
#define NX_(ix, iy) m->nextx[(size_t)((iy) - 1) * nx + ((ix) - 1)]
#define NY_(ix, iy) m->nexty[(size_t)((iy) - 1) * nx + ((ix) - 1)]
#define G(a, ix, iy) a[(size_t)((iy) - 1) * nx + ((ix) - 1)]
    /* CALC_REGION (no MPI): NSEQMAX = count of cells with NEXTX /= IMIS, :331-390 */
    int nseqmax = 0;
    for (size_t g = 0; g < ng; g++) if (m->nextx[g] != IMIS) nseqmax++;
    m->nseqmax = nseqmax;
    m->i1seqx = ialloc(nseqmax); m->i1seqy = ialloc(nseqmax); m->i1next = ialloc(nseqmax);
    m->i2vector = ialloc(ng);
    int upnmax = 0;
    for (int iy = 1; iy <= ny; iy++) for (int ix = 1; ix <= nx; ix++) {
        if (NX_(ix, iy) > 0) {
            int jx = NX_(ix, iy), jy = NY_(ix, iy);
            G(nupst, jx, jy) += 1;
            if (G(nupst, jx, jy) > upnmax) upnmax = G(nupst, jx, jy);
        }
    }
    int iseq = 0;
    for (int iy = 1; iy <= ny; iy++) for (int ix = 1; ix <= nx; ix++) {
        if (NX_(ix, iy) > 0 && G(nupst, ix, iy) == G(upnow, ix, iy)) {
            iseq++; m->i1seqx[iseq - 1] = ix; m->i1seqy[iseq - 1] = iy; G(m->i2vector, ix, iy) = iseq;
        }
    }
    int iseq1 = 1, iseq2 = iseq, again = 1, jseq = iseq2;
    while (again == 1) {
        again = 0; jseq = iseq2;
        for (int s = iseq1; s <= iseq2; s++) {
            int ix = m->i1seqx[s - 1], iy = m->i1seqy[s - 1];
            int jx = NX_(ix, iy), jy = NY_(ix, iy);
            G(upnow, jx, jy) += 1;
            if (G(upnow, jx, jy) == G(nupst, jx, jy) && NX_(jx, jy) > 0) {
                jseq++; m->i1seqx[jseq - 1] = jx; m->i1seqy[jseq - 1] = jy; G(m->i2vector, jx, jy) = jseq;
                again = 1;
            }
        }
        iseq1 = iseq2 + 1; iseq2 = jseq;
    }
    m->nseqriv = jseq;
    iseq = m->nseqriv;
    for (int iy = 1; iy <= ny; iy++) for (int ix = 1; ix <= nx; ix++) {
        if (NX_(ix, iy) < 0 && NX_(ix, iy) != IMIS) {
            iseq++; m->i1seqx[iseq - 1] = ix; m->i1seqy[iseq - 1] = iy; G(m->i2vector, ix, iy) = iseq;
        }
    }
    m->nseqall = iseq;
    if (m->nseqall != m->nseqmax) {
        snprintf(m->err, sizeof m->err, "NSEQALL(%d) /= NSEQMAX(%d): network has unreachable cells", m->nseqall, m->nseqmax);
        free(nupst); free(upnow); return -1;
    }
    for (int s = 0; s < m->nseqall; s++) {
        int ix = m->i1seqx[s], iy = m->i1seqy[s];
        if (NX_(ix, iy) > 0) m->i1next[s] = G(m->i2vector, NX_(ix, iy), NY_(ix, iy)) - 1;
        else m->i1next[s] = NX_(ix, iy);
    }
    /* upstream list, :515-522 */
    m->upnmax = upnmax;
    m->i1upst = ialloc((size_t)nseqmax * (upnmax ? upnmax : 1));
    m->i1upn = ialloc(nseqmax);
    for (int s = 0; s < m->nseqriv; s++) {
        int j = m->i1next[s];
        m->i1upn[j] += 1;
        m->i1upst[(size_t)j * upnmax + (m->i1upn[j] - 1)] = s;
    }
    free(nupst); free(upnow);
#undef NX_
#undef NY_
#undef G
    return 0;
}

/* ============================================================================ READ_BIFPARAM */
/* src/cmf_ctrl_maps_mod.F90:531-639 */
static int read_bifparam(orc_model *m) {
    FILE *f = fopen(m->cpthout, "r");
    if (!f) { snprintf(m->err, sizeof m->err, "cannot open %s", m->cpthout); return -1; }
    char line[4096];
    if (!fgets(line, sizeof line, f)) { fclose(f); return -1; }
    sscanf(line, "%d %d", &m->npthout, &m->npthlev);
    int P = m->npthout, Lp = m->npthlev;
    m->pth_upst = ialloc(P); m->pth_down = ialloc(P); m->pth_dst = dalloc(P);
    m->pth_elv = dalloc((size_t)P * Lp); m->pth_wth = dalloc((size_t)P * Lp); m->pth_man = dalloc(Lp);
    int *ocount = ialloc(m->nseqmax), *icount = ialloc(m->nseqmax);
    for (int p = 0; p < P; p++) {
        if (!fgets(line, sizeof line, f)) { fclose(f); snprintf(m->err, sizeof m->err, "short bifprm"); return -1; }
        char *s = line, *e;
        int ix = (int)strtol(s, &e, 10); s = e; int iy = (int)strtol(s, &e, 10); s = e;
        int jx = (int)strtol(s, &e, 10); s = e; int jy = (int)strtol(s, &e, 10); s = e;
        m->pth_dst[p] = strtod(s, &e); s = e;
        double pelv = strtod(s, &e); s = e; double pdph = strtod(s, &e); s = e;
        for (int l = 0; l < Lp; l++) { m->pth_wth[(size_t)l * P + p] = strtod(s, &e); s = e; }
        int up = m->i2vector[(size_t)(iy - 1) * m->nx + (ix - 1)];
        int dn = m->i2vector[(size_t)(jy - 1) * m->nx + (jx - 1)];
        m->pth_upst[p] = up; m->pth_down[p] = dn;          /* 1-based here; 0 = outside domain */
        if (up > 0 && dn > 0) { ocount[up - 1]++; icount[dn - 1]++; }
        for (int l = 1; l <= Lp; l++) {
            double pwth = m->pth_wth[(size_t)(l - 1) * P + p];
            double *elv = &m->pth_elv[(size_t)(l - 1) * P + p];
            if (l == 1) *elv = (pwth > 0) ? pelv - pdph : F(1.E20);
            else        *elv = (pwth > 0) ? (pelv + (double)l) - F(2.0) : F(1.E20);
        }
    }
    fclose(f);
    for (int l = 1; l <= Lp; l++) m->pth_man[l - 1] = (l == 1) ? m->pmanriv : m->pmanfld;
    int onmax = 0, inmax = 0;
    for (int s = 0; s < m->nseqmax; s++) { if (ocount[s] > onmax) onmax = ocount[s]; if (icount[s] > inmax) inmax = icount[s]; }
    m->onmax = onmax; m->inmax = inmax;
    m->i1p_out = ialloc((size_t)m->nseqmax * (onmax ? onmax : 1));
    m->i1p_inf = ialloc((size_t)m->nseqmax * (inmax ? inmax : 1));
    m->i1p_outn = ialloc(m->nseqmax); m->i1p_infn = ialloc(m->nseqmax);
    for (int p = 0; p < P; p++) {
        if (m->pth_upst[p] > 0 && m->pth_down[p] > 0) {
            int is = m->pth_upst[p] - 1, js = m->pth_down[p] - 1;
            m->i1p_outn[is]++; m->i1p_out[(size_t)is * onmax + m->i1p_outn[is] - 1] = p;
            m->i1p_infn[js]++; m->i1p_inf[(size_t)js * inmax + m->i1p_infn[js] - 1] = p;
        }
    }
    free(ocount); free(icount);
    return 0;
}

/* ============================================================================ TOPO_INIT */
/* src/cmf_ctrl_maps_mod.F90:651-736, READ_TOPO_BIN :745-849, SET_FLDSTG :969-999 */
static int topo_init(orc_model *m) {
    int N = m->nseqmax, L = m->nlfp;
    size_t ng = (size_t)m->nx * m->ny;
    float *r2 = (float *)malloc(ng * sizeof(float) * (size_t)(L > 1 ? L : 1));
    m->grarea = dalloc(N); m->elevtn = dalloc(N); m->nxtdst = dalloc(N); m->rivlen = dalloc(N);
    m->rivwth = dalloc(N); m->rivhgt = dalloc(N); m->fldhgt = dalloc((size_t)N * L); m->rivman = dalloc(N);
    m->dwnelv = dalloc(N); m->i2mask = ialloc(N);
    struct { const char *p; double *v; } maps[] = {
        {m->cgrarea, m->grarea}, {m->celevtn, m->elevtn}, {m->cnxtdst, m->nxtdst}, {m->crivlen, m->rivlen},
    };
    for (int k = 0; k < 4; k++) {
        if (read_f32_records(maps[k].p, r2, ng, 1)) { snprintf(m->err, sizeof m->err, "cannot read %s", maps[k].p); free(r2); return -1; }
        map_r2vec(m, r2, maps[k].v);
    }
    if (read_f32_records(m->cfldhgt, r2, ng, L)) { snprintf(m->err, sizeof m->err, "cannot read fldhgt"); free(r2); return -1; }
    for (int l = 0; l < L; l++) map_r2vec(m, r2 + (size_t)l * ng, m->fldhgt + (size_t)l * N);
    struct { const char *p; double *v; } maps2[] = { {m->crivhgt, m->rivhgt}, {m->crivwth, m->rivwth}, {m->crivman, m->rivman} };
    for (int k = 0; k < 3; k++) {
        if (read_f32_records(maps2[k].p, r2, ng, 1)) { snprintf(m->err, sizeof m->err, "cannot read %s", maps2[k].p); free(r2); return -1; }
        map_r2vec(m, r2, maps2[k].v);
    }
    free(r2);
    m->rivstomax = dalloc(N); m->rivelv = dalloc(N);
    for (int i = 0; i < N; i++) {
        m->rivstomax[i] = m->lfplain ? (m->rivlen[i] * m->rivwth[i]) * m->rivhgt[i] : F(1.E18);
        m->rivelv[i] = m->elevtn[i] - m->rivhgt[i];
    }
    /* SET_FLDSTG */
    m->fldstomax = dalloc((size_t)N * L); m->fldgrd = dalloc((size_t)N * L);
    m->dfrcinc = 1.0 / (double)L;
    for (int i = 0; i < N; i++) {
        double dstopre = m->rivstomax[i], dhgtpre = 0.0;
        double dwthinc = (m->grarea[i] * (1.0 / m->rivlen[i])) * m->dfrcinc;
        for (int I = 1; I <= L; I++) {
            double h = m->fldhgt[(size_t)(I - 1) * N + i];
            double dstonow = (m->rivlen[i] * (m->rivwth[i] + dwthinc * ((double)I - 0.5))) * (h - dhgtpre);
            m->fldstomax[(size_t)(I - 1) * N + i] = dstopre + dstonow;
            m->fldgrd[(size_t)(I - 1) * N + i] = (h - dhgtpre) * (1.0 / dwthinc);
            dstopre = m->fldstomax[(size_t)(I - 1) * N + i];
            dhgtpre = h;
        }
    }
    for (int i = 0; i < N; i++) m->dwnelv[i] = m->elevtn[i];
    return 0;
}

/* ============================================================================ LEVEE_INIT */
/* src/cmf_ctrl_levee_mod.F90:93-264 */
static int levee_init(orc_model *m) {
    int N = m->nseqmax, L = m->nlfp;
    size_t ng = (size_t)m->nx * m->ny;
    float *r2 = (float *)malloc(ng * sizeof(float));
    m->levhgt = dalloc(N); m->levfrc = dalloc(N);
    if (read_f32_records(m->clevhgt, r2, ng, 1)) { snprintf(m->err, sizeof m->err, "cannot read levhgt"); free(r2); return -1; }
    map_r2vec(m, r2, m->levhgt);
    if (read_f32_records(m->clevfrc, r2, ng, 1)) { snprintf(m->err, sizeof m->err, "cannot read levfrc"); free(r2); return -1; }
    map_r2vec(m, r2, m->levfrc);
    free(r2);
    m->bashgt = dalloc(N); m->levdst = dalloc(N);
    m->levbassto = dalloc(N); m->levtopsto = dalloc(N); m->levfilsto = dalloc(N);
    memset(m->fldstomax, 0, sizeof(double) * (size_t)N * L);
    memset(m->fldgrd, 0, sizeof(double) * (size_t)N * L);
    m->dfrcinc = 1.0 / (double)L;
    for (int i = 0; i < N; i++) {
        if (m->levhgt[i] <= 0.0) { m->levhgt[i] = 0.0; m->levfrc[i] = 1.0; }
        if (m->levfrc[i] >= 1.0 || m->levfrc[i] < 0.0) { m->levhgt[i] = 0.0; m->levfrc[i] = 1.0; }
        m->levfrc[i] = dmax(0.0, dmin(1.0, m->levfrc[i]));
    }
#define FSM(I) m->fldstomax[(size_t)((I) - 1) * N + i]
#define FGR(I) m->fldgrd[(size_t)((I) - 1) * N + i]
#define FHG(I) m->fldhgt[(size_t)((I) - 1) * N + i]
    for (int i = 0; i < N; i++) {
        double dsto_fil = m->rivstomax[i], dhgtpre = 0.0;
        double dwth_inc = (m->grarea[i] * (1.0 / m->rivlen[i])) * m->dfrcinc;
        for (int I = 1; I <= L; I++) {
            double dsto_add = (m->rivlen[i] * (m->rivwth[i] + dwth_inc * ((double)I - 0.5))) * (FHG(I) - dhgtpre);
            FSM(I) = dsto_fil + dsto_add;
            FGR(I) = (FHG(I) - dhgtpre) * (1.0 / dwth_inc);
            dsto_fil = FSM(I);
            dhgtpre = FHG(I);
        }
        if (m->levhgt[i] <= 0.0) {
            m->bashgt[i] = 1.E18; m->levdst[i] = 1.E18;
            m->levbassto[i] = 1.E18; m->levtopsto[i] = 1.E18; m->levfilsto[i] = 1.E18;
        } else {
            double dwth_fil, dwth_add, dhgtnow, dhgtdif;
            dsto_fil = m->rivstomax[i]; dhgtpre = 0.0; dwth_fil = 0.0;
            m->levdst[i] = (m->levfrc[i] * dwth_inc) * (double)L;
            int ilev = (int)(m->levfrc[i] * (double)L) + 1;
            if (ilev >= 2) { dsto_fil = FSM(ilev - 1); dhgtpre = FHG(ilev - 1); dwth_fil = dwth_inc * (double)(ilev - 1); }
            if (ilev <= L) {
                dwth_add = m->levdst[i] - dwth_fil;
                dhgtnow = dwth_add * FGR(ilev);
                m->bashgt[i] = dhgtnow + dhgtpre;
                m->levhgt[i] = dmax(m->levhgt[i], m->bashgt[i]);
                double dsto_add = (((dwth_add * F(0.5)) + dwth_fil) + m->rivwth[i]) * dhgtnow * m->rivlen[i];
                m->levbassto[i] = dsto_fil + dsto_add;
                dhgtdif = m->levhgt[i] - m->bashgt[i];
                m->levtopsto[i] = m->levbassto[i] + ((m->levdst[i] + m->rivwth[i]) * dhgtdif) * m->rivlen[i];
            } else {
                m->bashgt[i] = dhgtpre;
                m->levhgt[i] = dmax(m->levhgt[i], m->bashgt[i]);
                m->levbassto[i] = dsto_fil;
                dhgtdif = m->levhgt[i] - m->bashgt[i];
                m->levtopsto[i] = m->levbassto[i] + ((m->levdst[i] + m->rivwth[i]) * dhgtdif) * m->rivlen[i];
            }
            int I = 1;
            dsto_fil = m->rivstomax[i]; dwth_fil = m->rivwth[i]; dhgtpre = 0.0;
            while (m->levhgt[i] > FHG(I) && I <= L) {
                dsto_fil = FSM(I); dwth_fil = dwth_fil + dwth_inc; dhgtpre = FHG(I);
                I = I + 1; if (I > L) break;
            }
            if (I <= L) {
                dhgtnow = m->levhgt[i] - dhgtpre;
                dwth_add = dhgtnow / FGR(I);
                double dsto_add = ((dwth_add * 0.5) + dwth_fil) * dhgtnow * m->rivlen[i];
                m->levfilsto[i] = dsto_fil + dsto_add;
            } else {
                dhgtnow = m->levhgt[i] - dhgtpre;
                double dsto_add = (dwth_fil * dhgtnow) * m->rivlen[i];
                m->levfilsto[i] = dsto_fil + dsto_add;
            }
        }
    }
#undef FSM
#undef FGR
#undef FHG
    return 0;
}

/* ============================================================================ PROG_INIT */
/* src/cmf_ctrl_vars_mod.F90:28-176 (allocation + STORAGE_SEA_SURFACE), CMF_DIAG_INIT */
static void prog_diag_init(orc_model *m) {
    int N = m->nseqmax, PL = m->npthout * m->npthlev;
    m->runoff = dalloc(N); m->rofsub = dalloc(N); m->rivsto = dalloc(N); m->fldsto = dalloc(N);
    m->rivout = dalloc(N); m->fldout = dalloc(N); m->rivout_pre = dalloc(N); m->fldout_pre = dalloc(N);
    m->rivdph_pre = dalloc(N); m->fldsto_pre = dalloc(N); m->pthflw = dalloc(PL); m->pthflw_pre = dalloc(PL);
    m->gdwrtn = dalloc(N); m->damsto = dalloc(N); m->daminf = dalloc(N); m->levsto = dalloc(N);
    m->rivinf = dalloc(N); m->rivdph = dalloc(N); m->rivvel = dalloc(N); m->fldinf = dalloc(N);
    m->flddph = dalloc(N); m->fldfrc = dalloc(N); m->fldare = dalloc(N); m->pthout = dalloc(N); m->pthinf = dalloc(N);
    m->sfcelv = dalloc(N); m->outflw = dalloc(N); m->storge = dalloc(N); m->levdph = dalloc(N);
    m->pthflwsum = dalloc(m->npthout); m->stoout = dalloc(N); m->p_rivinf = dalloc(N); m->p_fldinf = dalloc(N);
    m->p_pthout = dalloc(N); m->rate = dalloc(N); m->sfcelv_pre = dalloc(N); m->dwnelv_pre = dalloc(N);
    m->flddph_pre = dalloc(N); m->sfcelv_lev = dalloc(N);
    m->rivout_a = dalloc(N); m->fldout_a = dalloc(N); m->outflw_a = dalloc(N); m->rivvel_a = dalloc(N);
    m->pthout_a = dalloc(N); m->gdwrtn_a = dalloc(N); m->runoff_a = dalloc(N); m->rofsub_a = dalloc(N);
    m->daminf_a = dalloc(N); m->storge_m = dalloc(N); m->outflw_m = dalloc(N); m->rivdph_m = dalloc(N);
    m->pthflw_a = dalloc(PL); m->pthflwsum_a = dalloc(m->npthout);
    m->rivout_o = dalloc(N); m->fldout_o = dalloc(N); m->outflw_o = dalloc(N); m->rivvel_o = dalloc(N);
    m->pthout_o = dalloc(N); m->gdwrtn_o = dalloc(N); m->runoff_o = dalloc(N); m->rofsub_o = dalloc(N);
    m->daminf_o = dalloc(N); m->storge_om = dalloc(N); m->outflw_om = dalloc(N); m->rivdph_om = dalloc(N);
    m->pthflw_o = dalloc(PL); m->nadd_out = 0.0;
    /* STORAGE_SEA_SURFACE, :129-176 */
    for (int i = m->nseqriv; i < m->nseqall; i++) {
        double dseaelv = m->dwnelv[i];
        double ddph = dmax(dseaelv - m->rivelv[i], 0.0);
        ddph = dmin(ddph, m->rivhgt[i]);
        m->rivsto[i] = (ddph * m->rivlen[i]) * m->rivwth[i];
        m->rivsto[i] = dmin(m->rivsto[i], m->rivstomax[i] * 1.0);
        m->rivdph_pre[i] = ddph;
    }
    for (int i = m->nseqriv - 1; i >= 0; i--) {
        int j = m->i1next[i];
        double dseaelv = m->rivelv[j] + m->rivdph_pre[j];
        double ddph = dmax(dseaelv - m->rivelv[i], 0.0);
        ddph = dmin(ddph, m->rivhgt[i]);
        m->rivsto[i] = (ddph * m->rivlen[i]) * m->rivwth[i];
        m->rivsto[i] = dmin(m->rivsto[i], m->rivstomax[i] * 1.0);
        m->rivdph_pre[i] = ddph;
    }
}

/* ============================================================================ DAMOUT_INIT */
/* src/cmf_ctrl_damout_mod.F90:123-308 (LRESTART=.FALSE., LDAMYBY handled for the file layout) */
static int damout_init(orc_model *m) {
    FILE *f = fopen(m->cdamfile, "r");
    if (!f) { snprintf(m->err, sizeof m->err, "cannot open %s", m->cdamfile); return -1; }
    char line[4096];
    if (!fgets(line, sizeof line, f)) { fclose(f); return -1; }
    int ndam = atoi(line);
    if (!fgets(line, sizeof line, f)) { fclose(f); return -1; }
    m->ndam = ndam;
    m->damseq = ialloc(ndam); m->damstat = ialloc(ndam); m->i1dam = ialloc(m->nseqmax);
    m->upreal = dalloc(ndam); m->r_volupa = dalloc(ndam); m->qf = dalloc(ndam); m->qn = dalloc(ndam);
    m->emevol = dalloc(ndam); m->fldvol = dalloc(ndam); m->convol = dalloc(ndam); m->norvol = dalloc(ndam);
    m->adjvol = dalloc(ndam); m->qa = dalloc(ndam);
    for (int d = 0; d < ndam; d++) { m->damseq[d] = IMIS; m->damstat[d] = IMIS; }
    int ndamx = 0;
    for (int d = 0; d < ndam; d++) {
        if (!fgets(line, sizeof line, f)) { fclose(f); snprintf(m->err, sizeof m->err, "short dam file"); return -1; }
        char *tok[16]; int nt = 0;
        for (char *p = strtok(line, ", \t\r\n"); p && nt < 16; p = strtok(NULL, ", \t\r\n")) tok[nt++] = p;
        if (nt < 12) { fclose(f); snprintf(m->err, sizeof m->err, "bad dam row"); return -1; }
        m->upreal[d] = strtod(tok[4], NULL);
        int ix = atoi(tok[5]), iy = atoi(tok[6]);
        double fldvol_mcm = strtod(tok[7], NULL), convol_mcm = strtod(tok[8], NULL);
        m->qn[d] = strtod(tok[10], NULL); m->qf[d] = strtod(tok[11], NULL);
        m->fldvol[d] = fldvol_mcm * 1.E6;
        m->convol[d] = convol_mcm * 1.E6;
        m->emevol[d] = m->convol[d] + m->fldvol[d] * 0.95;
        if (ix <= 0 || ix > m->nx || iy <= 0 || iy > m->ny) continue;
        int iseq = m->i2vector[(size_t)(iy - 1) * m->nx + (ix - 1)];
        if (iseq <= 0) continue;
        if (m->i1next[iseq - 1] == -9999) continue;
        ndamx++;
        m->damseq[d] = iseq - 1; m->damstat[d] = 2;
        m->i1dam[iseq - 1] = 1; m->i2mask[iseq - 1] = 2;
        if (m->ldamh22) {
            m->norvol[d] = m->convol[d] * 0.5;
            m->r_volupa[ndam - 1] = (m->fldvol[d] * F(1.E-6)) / m->upreal[d];   /* index NDAM as written */
        } else {
            double vyr = m->qn[d] * (double)(F(365.) * F(24.) * F(60.) * F(60.));
            double qsto = ((m->convol[d] * F(0.7)) + vyr / F(4.)) / (double)((float)180. * (float)24. * (float)60. * (float)60.);
            m->qn[d] = dmin(m->qn[d], qsto) * F(1.5);
            m->adjvol[d] = m->convol[d] + m->fldvol[d] * F(0.1);
            m->qa[d] = (m->qn[d] + m->qf[d]) * F(0.5);
        }
    }
    fclose(f);
    if (ndamx == 0) { snprintf(m->err, sizeof m->err, "none of the given dams allocated"); return -1; }
    for (int i = 0; i < m->nseqall; i++) {
        if (m->i1dam[i] <= 0 && m->i1next[i] >= 0) {
            int j = m->i1next[i];
            if (m->i1dam[j] == 1 || m->i1dam[j] == 11) { m->i1dam[i] = 10; m->i2mask[i] = 1; }
        }
        if (m->i1dam[i] == 1 && m->i1next[i] >= 0) {
            int j = m->i1next[i];
            if (m->i1dam[j] == 1 || m->i1dam[j] == 11) { m->i1dam[i] = 11; m->i2mask[i] = 2; }
        }
    }
    for (int i = 0; i < m->nseqmax; i++) m->damsto[i] = 0.0;
    for (int d = 0; d < ndam; d++) {
        if (m->damstat[d] == IMIS) continue;
        int s = m->damseq[d];
        if (m->damstat[d] == -1) m->damsto[s] = m->rivsto[s] + m->fldsto[s];
        else {
            m->damsto[s] = m->rivsto[s] + m->fldsto[s];
            if (m->damsto[s] < m->convol[d]) { m->damsto[s] = m->convol[d]; m->rivsto[s] = m->convol[d]; m->fldsto[s] = 0.0; }
        }
    }
    for (int i = 0; i < m->nseqall; i++) m->daminf[i] = 0.0;
    if (m->lpthout) {
        for (int p = 0; p < m->npthout; p++) {
            int up = m->pth_upst[p], dn = m->pth_down[p];
            if (up <= 0 || dn <= 0) continue;
            if (m->i1dam[up - 1] > 0 || m->i1dam[dn - 1] > 0)
                for (int l = 0; l < m->npthlev; l++) m->pth_elv[(size_t)l * m->npthout + p] = F(1.E20);
        }
    }
    return 0;
}

/* ============================================================================ FLDSTG */
/* CMF_CALC_FLDSTG_DEF, src/cmf_calc_fldstg_mod.F90:21-110 */
static void calc_fldstg_def(orc_model *m) {
    int N = m->nseqall, L = m->nlfp;
    m->glbstopre2 = m->glbstonew2 = m->glbrivsto = m->glbfldsto = m->glbfldare = 0.0;
    double sum = 0.0;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) reduction(+:sum)
#endif
    for (int i = 0; i < N; i++) {
        double pstoall = m->rivsto[i] + m->fldsto[i];
        double dstoall = pstoall;
        sum = sum + pstoall;
        if (pstoall > m->rivstomax[i]) {
            int I = 1;
            double dsto_fil = m->rivstomax[i], dwth_fil = m->rivwth[i], ddph_fil = 0.0, dsto_add, dwth_add;
            double dwth_inc = (m->grarea[i] / m->rivlen[i]) * m->dfrcinc;
            while (pstoall > m->fldstomax[(size_t)(I - 1) * N + i] && I <= L) {
                dsto_fil = m->fldstomax[(size_t)(I - 1) * N + i];
                dwth_fil = dwth_fil + dwth_inc;
                ddph_fil = ddph_fil + m->fldgrd[(size_t)(I - 1) * N + i] * dwth_inc;
                I = I + 1; if (I > L) break;
            }
            if (I > L) {
                dsto_add = dstoall - dsto_fil; dwth_add = 0.0;
                m->flddph[i] = ddph_fil + (dsto_add / dwth_fil) / m->rivlen[i];
            } else {
                double g = m->fldgrd[(size_t)(I - 1) * N + i];
                dsto_add = dstoall - dsto_fil;
                dwth_add = -dwth_fil + opow(dwth_fil * dwth_fil + ((2.0 * dsto_add) / m->rivlen[i]) / g, 0.5);
                m->flddph[i] = ddph_fil + g * dwth_add;
            }
            m->rivsto[i] = m->rivstomax[i] + (m->rivlen[i] * m->rivwth[i]) * m->flddph[i];
            m->rivsto[i] = dmin(m->rivsto[i], pstoall);
            m->rivdph[i] = (m->rivsto[i] / m->rivlen[i]) / m->rivwth[i];
            m->fldsto[i] = pstoall - m->rivsto[i];
            m->fldsto[i] = dmax(m->fldsto[i], 0.0);
            m->fldfrc[i] = ((-m->rivwth[i] + dwth_fil) + dwth_add) / (dwth_inc * (double)L);
            m->fldfrc[i] = dmax(m->fldfrc[i], 0.0);
            m->fldfrc[i] = dmin(m->fldfrc[i], 1.0);
            m->fldare[i] = m->grarea[i] * m->fldfrc[i];
        } else {
            m->rivsto[i] = pstoall;
            m->rivdph[i] = (dstoall / m->rivlen[i]) / m->rivwth[i];
            m->rivdph[i] = dmax(m->rivdph[i], 0.0);
            m->fldsto[i] = 0.0; m->flddph[i] = 0.0; m->fldfrc[i] = 0.0; m->fldare[i] = 0.0;
        }
    }
    m->glbstopre2 = sum;
    double s2 = 0, s3 = 0, s4 = 0, s5 = 0;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) reduction(+:s2,s3,s4,s5)
#endif
    for (int i = 0; i < N; i++) {
        m->sfcelv[i] = m->rivelv[i] + m->rivdph[i];
        m->storge[i] = m->rivsto[i] + m->fldsto[i];
        s2 = (s2 + m->rivsto[i]) + m->fldsto[i];
        s3 = s3 + m->rivsto[i];
        s4 = s4 + m->fldsto[i];
        s5 = s5 + m->fldare[i];
    }
    m->glbstonew2 = s2; m->glbrivsto = s3; m->glbfldsto = s4; m->glbfldare = s5;
}

/* CMF_LEVEE_FLDSTG, src/cmf_ctrl_levee_mod.F90:271-490 */
static void levee_fldstg(orc_model *m) {
    int N = m->nseqall, L = m->nlfp;
    double sum = 0.0;
#define FSM(I) m->fldstomax[(size_t)((I) - 1) * N + i]
#define FGR(I) m->fldgrd[(size_t)((I) - 1) * N + i]
#define FHG(I) m->fldhgt[(size_t)((I) - 1) * N + i]
#ifdef _OPENMP
#pragma omp parallel for schedule(static) reduction(+:sum)
#endif
    for (int i = 0; i < N; i++) {
        double pstoall = (m->rivsto[i] + m->fldsto[i]) + m->levsto[i];
        double dstoall = pstoall;
        sum = sum + pstoall;
        double dwth_inc = (m->grarea[i] / m->rivlen[i]) * m->dfrcinc;
        double dsto_add, dsto_fil, dwth_add, dwth_fil, ddph_fil, ddph_add;
        int I;
        if (dstoall > m->rivstomax[i]) {
            if (dstoall < m->levbassto[i]) {                                  /* case 1 */
                I = 1; dsto_fil = m->rivstomax[i]; dwth_fil = m->rivwth[i]; ddph_fil = 0.0;
                while (dstoall > FSM(I) && I <= L) {
                    dsto_fil = FSM(I); dwth_fil = dwth_fil + dwth_inc; ddph_fil = ddph_fil + FGR(I) * dwth_inc;
                    I = I + 1; if (I > L) break;
                }
                if (I <= L) {
                    dsto_add = dstoall - dsto_fil;
                    dwth_add = -dwth_fil + opow(dwth_fil * dwth_fil + ((2.0 * dsto_add) / m->rivlen[i]) / FGR(I), 0.5);
                    m->flddph[i] = ddph_fil + FGR(I) * dwth_add;
                } else {
                    dsto_add = dstoall - dsto_fil; dwth_add = 0.0;
                    m->flddph[i] = ddph_fil + (dsto_add / dwth_fil) / m->rivlen[i];
                }
                m->rivsto[i] = m->rivstomax[i] + (m->rivlen[i] * m->rivwth[i]) * m->flddph[i];
                m->rivdph[i] = (m->rivsto[i] / m->rivlen[i]) / m->rivwth[i];
                m->fldsto[i] = pstoall - m->rivsto[i];
                m->fldsto[i] = dmax(m->fldsto[i], 0.0);
                m->fldfrc[i] = ((-m->rivwth[i] + dwth_fil) + dwth_add) / (dwth_inc * (double)L);
                m->fldfrc[i] = dmax(m->fldfrc[i], 0.0);
                m->fldfrc[i] = dmin(m->fldfrc[i], 1.0);
                m->fldare[i] = m->grarea[i] * m->fldfrc[i];
                m->levsto[i] = 0.0; m->levdph[i] = 0.0;
            } else if (dstoall < m->levtopsto[i]) {                           /* case 2 */
                dsto_add = dstoall - m->levbassto[i];
                dwth_add = m->levdst[i] + m->rivwth[i];
                m->flddph[i] = m->bashgt[i] + (dsto_add / dwth_add) / m->rivlen[i];
                m->rivsto[i] = m->rivstomax[i] + (m->rivlen[i] * m->rivwth[i]) * m->flddph[i];
                m->rivdph[i] = (m->rivsto[i] / m->rivlen[i]) / m->rivwth[i];
                m->fldsto[i] = pstoall - m->rivsto[i];
                m->fldsto[i] = dmax(m->fldsto[i], 0.0);
                m->fldfrc[i] = m->levfrc[i];
                m->fldare[i] = m->grarea[i] * m->fldfrc[i];
                m->levsto[i] = 0.0; m->levdph[i] = 0.0;
            } else if (dstoall < m->levfilsto[i]) {                           /* case 3 */
                m->flddph[i] = m->levhgt[i];
                m->rivsto[i] = m->rivstomax[i] + (m->rivlen[i] * m->rivwth[i]) * m->flddph[i];
                m->rivdph[i] = (m->rivsto[i] / m->rivlen[i]) / m->rivwth[i];
                m->fldsto[i] = m->levtopsto[i] - m->rivsto[i];
                m->fldsto[i] = dmax(m->fldsto[i], 0.0);
                m->levsto[i] = (pstoall - m->rivsto[i]) - m->fldsto[i];
                m->levsto[i] = dmax(m->levsto[i], 0.0);
                int ilev = (int)(m->levfrc[i] * (double)L) + 1;
                dsto_fil = m->levtopsto[i]; dwth_fil = 0.0; ddph_fil = 0.0;
                I = ilev;
                while (I <= L) {
                    dsto_add = ((m->levdst[i] + m->rivwth[i]) * (m->levhgt[i] - FHG(I))) * m->rivlen[i];
                    if (dstoall < FSM(I) + dsto_add) break;
                    dsto_fil = FSM(I) + dsto_add;
                    dwth_fil = dwth_inc * (double)I - m->levdst[i];
                    ddph_fil = FHG(I) - m->bashgt[i];
                    I = I + 1; if (I > L) break;
                }
                if (I <= L) {
                    dsto_add = dstoall - dsto_fil;
                    dwth_add = -dwth_fil + opow(dwth_fil * dwth_fil + ((2.0 * dsto_add) / m->rivlen[i]) / FGR(I), 0.5);
                    ddph_add = dwth_add * FGR(I);
                    m->levdph[i] = (m->bashgt[i] + ddph_fil) + ddph_add;
                    m->fldfrc[i] = (dwth_fil + m->levdst[i]) / (dwth_inc * (double)L);
                    m->fldfrc[i] = dmax(m->fldfrc[i], 0.0);
                    m->fldfrc[i] = dmin(m->fldfrc[i], 1.0);
                    m->fldare[i] = m->grarea[i] * m->fldfrc[i];
                } else {
                    dsto_add = dstoall - dsto_fil;
                    ddph_add = (dsto_add / dwth_fil) / m->rivlen[i];
                    m->levdph[i] = (m->bashgt[i] + ddph_fil) + ddph_add;
                    m->fldfrc[i] = 1.0;
                    m->fldare[i] = m->grarea[i] * m->fldfrc[i];
                }
            } else {                                                          /* case 4 */
                I = 1; dsto_fil = m->rivstomax[i]; dwth_fil = m->rivwth[i]; ddph_fil = 0.0;
                while (dstoall > FSM(I) && I <= L) {
                    dsto_fil = FSM(I); dwth_fil = dwth_fil + dwth_inc; ddph_fil = ddph_fil + FGR(I) * dwth_inc;
                    I = I + 1; if (I > L) break;
                }
                if (I <= L) {
                    dsto_add = dstoall - dsto_fil;
                    dwth_add = -dwth_fil + opow(dwth_fil * dwth_fil + ((2.0 * dsto_add) / m->rivlen[i]) / FGR(I), 0.5);
                    m->flddph[i] = ddph_fil + FGR(I) * dwth_add;
                } else {
                    dsto_add = dstoall - dsto_fil; dwth_add = 0.0;
                    m->flddph[i] = ddph_fil + (dsto_add / dwth_fil) / m->rivlen[i];
                }
                m->fldfrc[i] = ((-m->rivwth[i] + dwth_fil) + dwth_add) / (dwth_inc * (double)L);
                m->fldare[i] = m->grarea[i] * m->fldfrc[i];
                m->rivsto[i] = m->rivstomax[i] + (m->rivlen[i] * m->rivwth[i]) * m->flddph[i];
                m->rivdph[i] = (m->rivsto[i] / m->rivlen[i]) / m->rivwth[i];
                dsto_add = ((m->flddph[i] - m->levhgt[i]) * (m->levdst[i] + m->rivwth[i])) * m->rivlen[i];
                m->fldsto[i] = (m->levtopsto[i] + dsto_add) - m->rivsto[i];
                m->fldsto[i] = dmax(m->fldsto[i], 0.0);
                m->levsto[i] = (pstoall - m->rivsto[i]) - m->fldsto[i];
                m->levsto[i] = dmax(m->levsto[i], 0.0);
                m->levdph[i] = m->flddph[i];
            }
        } else {                                                              /* case 0 */
            m->rivsto[i] = pstoall;
            m->rivdph[i] = (dstoall / m->rivlen[i]) / m->rivwth[i];
            m->rivdph[i] = dmax(m->rivdph[i], 0.0);
            m->fldsto[i] = 0.0; m->flddph[i] = 0.0; m->fldfrc[i] = 0.0; m->fldare[i] = 0.0;
            m->levsto[i] = 0.0; m->levdph[i] = 0.0;
        }
    }
#undef FSM
#undef FGR
#undef FHG
    m->glbstopre2 = sum;
    double s2 = 0, s3 = 0, s4 = 0, s5 = 0, s6 = 0;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) reduction(+:s2,s3,s4,s5,s6)
#endif
    for (int i = 0; i < N; i++) {
        m->sfcelv[i] = m->rivelv[i] + m->rivdph[i];
        m->storge[i] = (m->rivsto[i] + m->fldsto[i]) + m->levsto[i];
        s2 = ((s2 + m->rivsto[i]) + m->fldsto[i]) + m->levsto[i];
        s3 = s3 + m->rivsto[i]; s4 = s4 + m->fldsto[i]; s5 = s5 + m->levsto[i]; s6 = s6 + m->fldare[i];
    }
    m->glbstonew2 = s2; m->glbrivsto = s3; m->glbfldsto = s4; m->glblevsto = s5; m->glbfldare = s6;
}

/* CMF_PHYSICS_FLDSTG, src/cmf_ctrl_physics_mod.F90:288-305 */
static void physics_fldstg(orc_model *m) {
    if (m->llevee) levee_fldstg(m); else calc_fldstg_def(m);
}

/* ============================================================================ OUTFLW */
/* CMF_CALC_OUTFLW, src/cmf_calc_outflw_mod.F90:32-185 */
static void calc_outflw(orc_model *m, double DT) {
    int N = m->nseqall, R = m->nseqriv;
    const double gdt = m->pgrv * DT;
    OMP_FOR
    for (int i = 0; i < N; i++) {
        m->sfcelv[i] = m->rivelv[i] + m->rivdph[i];
        m->sfcelv_pre[i] = m->rivelv[i] + m->rivdph_pre[i];
        m->flddph_pre[i] = dmax(m->rivdph_pre[i] - m->rivhgt[i], 0.0);
    }
    OMP_FOR
    for (int i = 0; i < R; i++) {
        int j = m->i1next[i];
        m->dwnelv[i] = m->sfcelv[j];
        m->dwnelv_pre[i] = m->sfcelv_pre[j];
    }
    OMP_FOR
    for (int i = 0; i < R; i++) {
        double dsfc = dmax(m->sfcelv[i], m->dwnelv[i]);
        double dslp = (m->sfcelv[i] - m->dwnelv[i]) * (1.0 / m->nxtdst[i]);
        double dflw = dsfc - m->rivelv[i];
        double dare = dmax(m->rivwth[i] * dflw, 1.E-10);
        double dsfc_pr = dmax(m->sfcelv_pre[i], m->dwnelv_pre[i]);
        double dflw_pr = dsfc_pr - m->rivelv[i];
        double dflw_im = dmax(opow(dflw * dflw_pr, 0.5), 1.E-6);
        double dout_pr = m->rivout_pre[i] * (1.0 / m->rivwth[i]);
        double dout = (m->rivwth[i] * (dout_pr + (gdt * dflw_im) * dslp))
                    * (1.0 / (1.0 + ((gdt * (m->rivman[i] * m->rivman[i])) * fabs(dout_pr)) * opow(dflw_im, -7.0 / 3.0)));
        double dvel = m->rivout[i] * (1.0 / dare);
        int mask = (dflw_im > F(1.E-5) && dare > F(1.E-5));
        m->rivout[i] = mask ? dout : 0.0;
        m->rivvel[i] = mask ? dvel : 0.0;
    }
    if (m->lfldout) {
        OMP_FOR
        for (int i = 0; i < R; i++) {
            double dfsto = m->fldsto[i];
            double dsfc = dmax(m->sfcelv[i], m->dwnelv[i]);
            double dslp = (m->sfcelv[i] - m->dwnelv[i]) * (1.0 / m->nxtdst[i]);
            dslp = dmax(-0.005, dmin(0.005, dslp));
            double dflw = dmax(dsfc - m->elevtn[i], 0.0);
            double dare = dfsto * (1.0 / m->rivlen[i]);
            dare = dmax(dare - m->flddph[i] * m->rivwth[i], 0.0);
            double dsfc_pr = dmax(m->sfcelv_pre[i], m->dwnelv_pre[i]);
            double dflw_pr = dsfc_pr - m->elevtn[i];
            double dflw_im = dmax(opow(dmax(dflw * dflw_pr, 0.0), 0.5), 1.E-6);
            double dare_pr = m->fldsto_pre[i] * (1.0 / m->rivlen[i]);
            dare_pr = dmax(dare_pr - m->flddph_pre[i] * m->rivwth[i], 1.E-6);
            double dare_im = dmax(opow(dare * dare_pr, 0.5), 1.E-6);
            double dout_pr = m->fldout_pre[i];
            double dout = (dout_pr + (gdt * dare_im) * dslp)
                        * (1.0 / (1.0 + (((gdt * (m->pmanfld * m->pmanfld)) * fabs(dout_pr)) * opow(dflw_im, -4.0 / 3.0)) * (1.0 / dare_im)));
            int mask = (dflw_im > 1.E-5 && dare > 1.E-5);
            m->fldout[i] = mask ? dout : 0.0;
            dout = m->fldout[i];
            mask = (m->fldout[i] * m->rivout[i] > 0.0);
            m->fldout[i] = mask ? dout : 0.0;
        }
    }
    OMP_FOR
    for (int i = R; i < N; i++) {
        double dslp = (m->sfcelv[i] - m->dwnelv[i]) * (1.0 / m->pdstmth);
        double dflw = m->rivdph[i];
        double dare = m->rivwth[i] * dflw;
        dare = dmax(dare, 1.E-10);
        double dflw_pr = m->rivdph_pre[i];
        double dflw_im = dmax(opow(dflw * dflw_pr, 0.5), 1.E-6);
        double dout_pr = m->rivout_pre[i] * (1.0 / m->rivwth[i]);
        double dout = (m->rivwth[i] * (dout_pr + (gdt * dflw_im) * dslp))
                    * (1.0 / (1.0 + ((gdt * (m->rivman[i] * m->rivman[i])) * fabs(dout_pr)) * opow(dflw_im, -7.0 / 3.0)));
        double dvel = m->rivout[i] * (1.0 / dare);
        int mask = (dflw_im > F(1.E-5) && dare > F(1.E-5));
        m->rivout[i] = mask ? dout : 0.0;
        m->rivvel[i] = mask ? dvel : 0.0;
    }
    if (m->lfldout) {
        OMP_FOR
        for (int i = R; i < N; i++) {
            double dfsto = m->fldsto[i];
            double dslp = (m->sfcelv[i] - m->dwnelv[i]) * (1.0 / m->pdstmth);
            dslp = dmax(-0.005, dmin(0.005, dslp));
            double dflw = m->sfcelv[i] - m->elevtn[i];
            double dare = dmax(dfsto * (1.0 / m->rivlen[i]) - m->flddph[i] * m->rivwth[i], 0.0);
            double dflw_pr = m->sfcelv_pre[i] - m->elevtn[i];
            double dflw_im = dmax(opow(dmax(dflw * dflw_pr, 0.0), 0.5), 1.E-6);
            double dare_pr = dmax(m->fldsto_pre[i] * (1.0 / m->rivlen[i]) - m->flddph_pre[i] * m->rivwth[i], 1.E-6);
            double dare_im = dmax(opow(dare * dare_pr, 0.5), 1.E-6);
            double dout_pr = m->fldout_pre[i];
            double dout = (dout_pr + (gdt * dare_im) * dslp)
                        * (1.0 / (1.0 + (((gdt * (m->pmanfld * m->pmanfld)) * fabs(dout_pr)) * opow(dflw_im, -4.0 / 3.0)) * (1.0 / dare_im)));
            int mask = (dflw_im > F(1.E-5) && dare > F(1.E-5));
            m->fldout[i] = mask ? dout : 0.0;
            dout = m->fldout[i];
            mask = (m->fldout[i] * m->rivout[i] > 0.0);
            m->fldout[i] = mask ? dout : 0.0;
        }
    }
    OMP_FOR
    for (int i = 0; i < R; i++) {
        double dout = dmax((-m->rivout[i] - m->fldout[i]) * DT, F(1.E-10));
        double rate = dmin((0.05 * m->storge[i]) / dout, 1.0);
        m->rivout[i] = m->rivout[i] * rate;
        m->fldout[i] = m->fldout[i] * rate;
    }
}

/* ============================================================================ PTHOUT */
/* CMF_CALC_PTHOUT, src/cmf_calc_pthout_mod.F90:20-97 */
static void calc_pthout(orc_model *m, double DT) {
    int N = m->nseqall, P = m->npthout, Lp = m->npthlev;
    const double gdt = m->pgrv * DT;
    OMP_FOR
    for (int i = 0; i < N; i++) m->sfcelv_pre[i] = m->rivelv[i] + m->rivdph_pre[i];
    for (size_t k = 0; k < (size_t)P * Lp; k++) m->pthflw[k] = 0.0;
    OMP_FOR
    for (int p = 0; p < P; p++) {
        int up = m->pth_upst[p], dn = m->pth_down[p];
        if (up <= 0 || dn <= 0) continue;
        up -= 1; dn -= 1;
        if (m->i2mask[up] > 0 || m->i2mask[dn] > 0) continue;
        double dslp = (m->sfcelv[up] - m->sfcelv[dn]) / m->pth_dst[p];
        dslp = dmax(-0.005, dmin(0.005, dslp));
        for (int l = 0; l < Lp; l++) {
            double elv = m->pth_elv[(size_t)l * P + p];
            double dflw = dmax(m->sfcelv[up], m->sfcelv[dn]) - elv;
            dflw = dmax(dflw, 0.0);
            double dflw_pr = dmax(m->sfcelv_pre[up], m->sfcelv_pre[dn]) - elv;
            dflw_pr = dmax(dflw_pr, 0.0);
            double dflw_im = opow(dflw * dflw_pr, 0.5);
            dflw_im = dmax(dflw_im, opow(dflw * 0.01, 0.5));
            if (dflw_im > 1.E-5) {
                double wth = m->pth_wth[(size_t)l * P + p];
                double dout_pr = m->pthflw_pre[(size_t)l * P + p] / wth;
                m->pthflw[(size_t)l * P + p] = (wth * (dout_pr + (gdt * dflw_im) * dslp))
                    / (1.0 + ((gdt * (m->pth_man[l] * m->pth_man[l])) * fabs(dout_pr)) * opow(dflw_im, -7.0 / 3.0));
            } else {
                m->pthflw[(size_t)l * P + p] = 0.0;
            }
        }
        m->pthflwsum[p] = 0.0;
    }
    for (int p = 0; p < P; p++) {
        double s = 0.0;
        for (int l = 0; l < Lp; l++) s = s + m->pthflw[(size_t)l * P + p];
        m->pthflwsum[p] = s;
    }
    for (int p = 0; p < P; p++) {
        if (m->pthflwsum[p] != 0.0) {
            int up = m->pth_upst[p] - 1, dn = m->pth_down[p] - 1;
            double rate = (0.05 * dmin(m->storge[up], m->storge[dn])) / fabs(m->pthflwsum[p] * DT);
            rate = dmin(rate, 1.0);
            for (int l = 0; l < Lp; l++) m->pthflw[(size_t)l * P + p] = m->pthflw[(size_t)l * P + p] * rate;
            m->pthflwsum[p] = m->pthflwsum[p] * rate;
        }
    }
}

/* CMF_LEVEE_OPT_PTHOUT, src/cmf_ctrl_levee_mod.F90:497-603 */
static void levee_opt_pthout(orc_model *m, double DT) {
    int N = m->nseqall, P = m->npthout, Lp = m->npthlev;
    const double gdt = m->pgrv * DT;
    OMP_FOR
    for (int i = 0; i < N; i++) {
        m->sfcelv_lev[i] = m->sfcelv[i];
        if (m->levfrc[i] < 1.0) m->sfcelv_lev[i] = dmin(m->elevtn[i] + m->levdph[i], m->sfcelv[i]);
        m->sfcelv_pre[i] = m->rivelv[i] + m->rivdph_pre[i];
    }
    for (size_t k = 0; k < (size_t)P * Lp; k++) m->pthflw[k] = 0.0;
    OMP_FOR
    for (int p = 0; p < P; p++) {
        int up = m->pth_upst[p], dn = m->pth_down[p];
        if (up <= 0 || dn <= 0) continue;
        up -= 1; dn -= 1;
        if (m->i2mask[up] == 1 || m->i2mask[dn] == 1) continue;
        double dslp = (m->sfcelv[up] - m->sfcelv[dn]) / m->pth_dst[p];
        dslp = dmax(-0.005, dmin(0.005, dslp));
        {
            int l = 0;
            double elv = m->pth_elv[(size_t)l * P + p];
            double dflw = dmax(m->sfcelv[up], m->sfcelv[dn]) - elv;
            dflw = dmax(dflw, 0.0);
            double dflw_pr = dmax(m->sfcelv_pre[up], m->sfcelv_pre[dn]) - elv;
            dflw_pr = dmax(dflw_pr, 0.0);
            double dflw_im = opow(dflw * dflw_pr, 0.5);
            if (dflw_im <= 0.0) dflw_im = dflw;
            if (dflw_im > 1.E-5) {
                double wth = m->pth_wth[(size_t)l * P + p];
                double dout_pr = m->pthflw_pre[(size_t)l * P + p] / wth;
                m->pthflw[(size_t)l * P + p] = (wth * (dout_pr + (gdt * dflw_im) * dslp))
                    / (1.0 + ((gdt * (m->pth_man[l] * m->pth_man[l])) * fabs(dout_pr)) * opow(dflw_im, -7.0 / 3.0));
            } else {
                m->pthflw[(size_t)l * P + p] = 0.0;
            }
        }
        if (Lp <= 1) continue;
        dslp = (m->sfcelv[up] - m->sfcelv[dn]) / m->pth_dst[p];
        dslp = dmax(-0.005, dmin(0.005, dslp));
        for (int l = 1; l < Lp; l++) {
            double elv = m->pth_elv[(size_t)l * P + p];
            double dflw = dmax(m->sfcelv_lev[up], m->sfcelv_lev[dn]) - elv;
            dflw = dmax(dflw, 0.0);
            double dflw_im = dflw;
            if (dflw_im > 1.E-5) {
                double wth = m->pth_wth[(size_t)l * P + p];
                double dout_pr = m->pthflw_pre[(size_t)l * P + p] * (1.0 / wth);
                m->pthflw[(size_t)l * P + p] = (wth * (dout_pr + (gdt * dflw_im) * dslp))
                    / (1.0 + ((gdt * (m->pth_man[l] * m->pth_man[l])) * fabs(dout_pr)) * opow(dflw_im, -7.0 / 3.0));
            } else {
                m->pthflw[(size_t)l * P + p] = 0.0;
            }
        }
        m->pthflwsum[p] = 0.0;
    }
    for (int p = 0; p < P; p++) {
        double s = 0.0;
        for (int l = 0; l < Lp; l++) s = s + m->pthflw[(size_t)l * P + p];
        m->pthflwsum[p] = s;
    }
    for (int p = 0; p < P; p++) {
        if (m->pthflwsum[p] != 0.0) {
            int up = m->pth_upst[p] - 1, dn = m->pth_down[p] - 1;
            double rate = (0.05 * dmin(m->storge[up], m->storge[dn])) / fabs(m->pthflwsum[p] * DT);
            rate = dmin(rate, 1.0);
            for (int l = 0; l < Lp; l++) m->pthflw[(size_t)l * P + p] = m->pthflw[(size_t)l * P + p] * rate;
            m->pthflwsum[p] = m->pthflwsum[p] * rate;
        }
    }
}

/* ============================================================================ DAMOUT */
/* CMF_DAMOUT_CALC + UPDATE_INFLOW, src/cmf_ctrl_damout_mod.F90:316-498 */
static void damout_calc(orc_model *m, double DT) {
    int N = m->nseqall, R = m->nseqriv;
    const double p23 = F(2. / 3.);
    for (int i = 0; i < N; i++) {
        if (m->i1dam[i] > 0) { m->rivout[i] = 0.0; m->fldout[i] = 0.0; m->daminf[i] = m->runoff[i]; }
    }
    for (int i = 0; i < N; i++) {            /* serial: the -DNoAtom_CMF order */
        if (m->i1dam[i] == 10 || m->i1dam[i] == 11) {
            int j = m->i1next[i];
            m->daminf[j] = (m->daminf[j] + m->rivout_pre[i]) + m->fldout_pre[i];
        }
    }
    for (int i = 0; i < R; i++) {
        if (m->i1dam[i] == 10) {
            int j = m->i1next[i];
            double dslope = (m->elevtn[i] - m->elevtn[j]) * (1.0 / m->nxtdst[i]);
            dslope = dmax(dslope, m->pminslp);
            double dvel = ((1.0 / m->rivman[i]) * opow(dslope, 0.5)) * opow(m->rivdph[i], p23);
            double darea = m->rivwth[i] * m->rivdph[i];
            m->rivvel[i] = dvel;
            m->rivout[i] = darea * dvel;
            m->rivout[i] = dmin(m->rivout[i], m->rivsto[i] / DT);
            double dslope_f = dmin(0.005, dslope);
            double dvel_f = ((1.0 / m->pmanfld) * opow(dslope_f, 0.5)) * opow(m->flddph[i], p23);
            double dare_f = m->fldsto[i] * (1.0 / m->rivlen[i]);
            dare_f = dmax(dare_f - m->flddph[i] * m->rivwth[i], 0.0);
            m->fldout[i] = dare_f * dvel_f;
            m->fldout[i] = dmin(m->fldout[i], m->fldsto[i] / DT);
        }
    }
    static double damoutflw = 0.0;   /* SAVE variable of the reference */
    for (int d = 0; d < m->ndam; d++) {
        if (m->damstat[d] <= 0) continue;
        int s = m->damseq[d];
        double damvol = m->damsto[s], daminflow = m->daminf[s], tmp;
        if (m->ldamh22) {
            if (damvol <= m->norvol[d]) damoutflw = m->qn[d] * (damvol / m->convol[d]);
            else if (m->norvol[d] < damvol && damvol <= m->convol[d]) {
                if (m->qf[d] <= daminflow)
                    damoutflw = m->qn[d] * F(0.5) + ((damvol - m->norvol[d]) / (m->convol[d] - m->norvol[d])) * (m->qf[d] - m->qn[d]);
                else {
                    double r = (damvol - m->norvol[d]) / (m->emevol[d] - m->norvol[d]);
                    damoutflw = m->qn[d] * F(0.5) + (r * r) * (m->qf[d] - m->qn[d]);
                }
            } else if (m->convol[d] < damvol && damvol < m->emevol[d]) {
                if (m->qf[d] <= daminflow)
                    damoutflw = m->qf[d] + ((dmax(F(1.) - m->r_volupa[d] / F(0.2), 0.0) * (damvol - m->convol[d])) / (m->emevol[d] - m->convol[d])) * (daminflow - m->qf[d]);
                else {
                    double r = (damvol - m->norvol[d]) / (m->emevol[d] - m->norvol[d]);
                    damoutflw = m->qn[d] * F(0.5) + (r * r) * (m->qf[d] - m->qn[d]);
                }
            } else damoutflw = dmax(daminflow, m->qf[d]);
        } else {
            if (damvol <= m->convol[d]) {
                damoutflw = m->qn[d] * opow(damvol / m->convol[d], F(0.5));
            } else if (damvol > m->convol[d] && damvol <= m->adjvol[d]) {
                damoutflw = m->qn[d] + opow((damvol - m->convol[d]) / (m->adjvol[d] - m->convol[d]), F(3.0)) * (m->qa[d] - m->qn[d]);
            } else if (damvol > m->adjvol[d] && damvol <= m->emevol[d]) {
                if (daminflow >= m->qf[d]) {
                    damoutflw = m->qn[d] + ((damvol - m->convol[d]) / (m->emevol[d] - m->convol[d])) * (daminflow - m->qn[d]);
                    tmp = m->qa[d] + opow((damvol - m->adjvol[d]) / (m->emevol[d] - m->adjvol[d]), F(0.1)) * (m->qf[d] - m->qa[d]);
                    damoutflw = dmax(damoutflw, tmp);
                } else {
                    damoutflw = m->qa[d] + opow((damvol - m->adjvol[d]) / (m->emevol[d] - m->adjvol[d]), F(0.1)) * (m->qf[d] - m->qa[d]);
                }
            } else if (damvol > m->emevol[d]) {
                damoutflw = (daminflow >= m->qf[d]) ? daminflow : m->qf[d];
            }
        }
        damoutflw = dmin(dmin(damoutflw, damvol / DT), (m->rivsto[s] + m->fldsto[s]) / DT);
        damoutflw = dmax(damoutflw, 0.0);
        m->rivout[s] = damoutflw;
        m->fldout[s] = 0.0;
    }
}

/* CMF_DAMOUT_WATBAL, src/cmf_ctrl_damout_mod.F90:504-542 */
static void damout_watbal(orc_model *m, double DT) {
    double s0 = 0, s1 = 0, si = 0, so = 0;
    for (int d = 0; d < m->ndam; d++) {
        if (m->damstat[d] == IMIS) continue;
        int s = m->damseq[d];
        double inflow = (m->rivinf[s] + m->fldinf[s]) + m->runoff[s];
        double outflw = m->rivout[s] + m->fldout[s];
        s0 = s0 + m->damsto[s];
        si = si + inflow * DT;
        so = so + outflw * DT;
        m->damsto[s] = (m->damsto[s] + inflow * DT) - outflw * DT;
        s1 = s1 + m->damsto[s];
    }
    m->dam_miss = ((s0 - s1) + si) - so;
}

/* ============================================================================ INFLOW */
/* CMF_CALC_INFLOW_LSPAMAT, src/cmf_calc_outflw_mod.F90:386-546 */
static void calc_inflow_lspamat(orc_model *m, double DT) {
    int N = m->nseqall, R = m->nseqriv, P = m->npthout, Lp = m->npthlev;
    OMP_FOR
    for (int i = 0; i < N; i++) { m->p_rivinf[i] = 0.0; m->p_fldinf[i] = 0.0; m->p_pthout[i] = 0.0; m->stoout[i] = 0.0; }
    OMP_FOR
    for (int i = 0; i < N; i++) {
        double s = dmax(m->rivout[i], 0.0) + dmax(m->fldout[i], 0.0);
        for (int k = 0; k < m->i1upn[i]; k++) {
            int j = m->i1upst[(size_t)i * m->upnmax + k];
            s = (s + dmax(-m->rivout[j], 0.0)) + dmax(-m->fldout[j], 0.0);
        }
        m->stoout[i] = s * DT;
    }
    if (m->lpthout) {
        OMP_FOR
        for (int i = 0; i < N; i++) {
            for (int k = 0; k < m->i1p_outn[i]; k++) {
                int p = m->i1p_out[(size_t)i * m->onmax + k];
                m->stoout[i] = m->stoout[i] + dmax(m->pthflwsum[p], 0.0) * DT;
            }
            for (int k = 0; k < m->i1p_infn[i]; k++) {
                int p = m->i1p_inf[(size_t)i * m->inmax + k];
                m->stoout[i] = m->stoout[i] + dmax(-m->pthflwsum[p], 0.0) * DT;
            }
        }
    }
    OMP_FOR
    for (int i = 0; i < N; i++) {
        double dout = dmax(m->stoout[i], 1.E-10);
        double dsto = m->rivsto[i] + m->fldsto[i];
        m->rate[i] = dmin(dsto / dout, 1.0);
    }
    OMP_FOR
    for (int i = 0; i < R; i++) {
        int j = m->i1next[i];
        if (m->rivout[i] > 0.0) { m->rivout[i] = m->rivout[i] * m->rate[i]; m->fldout[i] = m->fldout[i] * m->rate[i]; }
        else { m->rivout[i] = m->rivout[i] * m->rate[j]; m->fldout[i] = m->fldout[i] * m->rate[j]; }
    }
    OMP_FOR
    for (int i = R; i < N; i++) { m->rivout[i] = m->rivout[i] * m->rate[i]; m->fldout[i] = m->fldout[i] * m->rate[i]; }
    OMP_FOR
    for (int i = 0; i < N; i++) {
        for (int k = 0; k < m->i1upn[i]; k++) {
            int j = m->i1upst[(size_t)i * m->upnmax + k];
            m->p_rivinf[i] = m->p_rivinf[i] + m->rivout[j];
            m->p_fldinf[i] = m->p_fldinf[i] + m->fldout[j];
        }
    }
    if (m->lpthout) {
        OMP_FOR
        for (int p = 0; p < P; p++) {
            int up = m->pth_upst[p], dn = m->pth_down[p];
            if (up <= 0 || dn <= 0) continue;
            up -= 1; dn -= 1;
            if (m->i2mask[up] > 0 || m->i2mask[dn] > 0) continue;
            for (int l = 0; l < Lp; l++) {
                double *f = &m->pthflw[(size_t)l * P + p];
                if (*f >= 0.0) *f = *f * m->rate[up]; else *f = *f * m->rate[dn];
            }
            if (m->pthflwsum[p] >= 0.0) m->pthflwsum[p] = m->pthflwsum[p] * m->rate[up];
            else m->pthflwsum[p] = m->pthflwsum[p] * m->rate[dn];
        }
        OMP_FOR
        for (int i = 0; i < N; i++) {
            for (int k = 0; k < m->i1p_outn[i]; k++) m->p_pthout[i] = m->p_pthout[i] + m->pthflwsum[m->i1p_out[(size_t)i * m->onmax + k]];
            for (int k = 0; k < m->i1p_infn[i]; k++) m->p_pthout[i] = m->p_pthout[i] - m->pthflwsum[m->i1p_inf[(size_t)i * m->inmax + k]];
        }
    }
    OMP_FOR
    for (int i = 0; i < N; i++) { m->rivinf[i] = m->p_rivinf[i]; m->fldinf[i] = m->p_fldinf[i]; m->pthout[i] = m->p_pthout[i]; }
}

/* ============================================================================ STONXT */
/* CMF_CALC_STONXT, src/cmf_calc_stonxt_mod.F90:20-136 (no groundwater delay, no LROSPLIT) */
static void calc_stonxt(orc_model *m, double DT) {
    int N = m->nseqall;
    double a = 0, b = 0, c = 0, d = 0, e = 0;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) reduction(+:a,b,c,d,e)
#endif
    for (int i = 0; i < N; i++) {
        a = (a + m->rivsto[i]) + m->fldsto[i];
        b = (b + m->rivinf[i] * DT) + m->fldinf[i] * DT;
        c = ((c + m->rivout[i] * DT) + m->fldout[i] * DT) + m->pthout[i] * DT;
        m->rivsto[i] = (m->rivsto[i] + m->rivinf[i] * DT) - m->rivout[i] * DT;
        if (m->rivsto[i] < 0.0) { m->fldsto[i] = m->fldsto[i] + m->rivsto[i]; m->rivsto[i] = 0.0; }
        m->fldsto[i] = ((m->fldsto[i] + m->fldinf[i] * DT) - m->fldout[i] * DT) - m->pthout[i] * DT;
        if (m->fldsto[i] < 0.0) { m->rivsto[i] = dmax(m->rivsto[i] + m->fldsto[i], 0.0); m->fldsto[i] = 0.0; }
        d = (d + m->rivsto[i]) + m->fldsto[i];
        m->outflw[i] = m->rivout[i] + m->fldout[i];
        double drivrof = ((m->runoff[i] + m->gdwrtn[i]) * (1.0 - m->fldfrc[i])) * DT;
        double dfldrof = ((m->runoff[i] + m->gdwrtn[i]) * m->fldfrc[i]) * DT;
        m->rivsto[i] = m->rivsto[i] + drivrof;
        m->fldsto[i] = m->fldsto[i] + dfldrof;
        m->storge[i] = m->rivsto[i] + m->fldsto[i];
        if (m->llevee) m->storge[i] = m->storge[i] + m->levsto[i];
        e = e + m->storge[i];
    }
    m->glbstopre = a; m->glbrivinf = b; m->glbrivout = c; m->glbstonxt = d; m->glbstonew = e;
}

/* ============================================================================ DIAG */
/* src/cmf_calc_diag_mod.F90:50-221 */
static void diag_reset_adpstp(orc_model *m) {
    int N = m->nseqmax, PL = m->npthout * m->npthlev;
    m->nadd_adp = 0.0;
    for (int i = 0; i < N; i++) {
        m->rivout_a[i] = m->fldout_a[i] = m->outflw_a[i] = m->rivvel_a[i] = m->pthout_a[i] = 0.0;
        m->gdwrtn_a[i] = m->runoff_a[i] = m->rofsub_a[i] = 0.0;
        m->storge_m[i] = m->outflw_m[i] = m->rivdph_m[i] = 0.0;
        m->daminf_a[i] = 0.0;
    }
    for (int k = 0; k < PL; k++) m->pthflw_a[k] = 0.0;
    for (int p = 0; p < m->npthout; p++) m->pthflwsum_a[p] = 0.0;
}
static void diag_avemax_adpstp(orc_model *m, double DT) {
    int N = m->nseqmax, PL = m->npthout * m->npthlev;
    m->nadd_adp = m->nadd_adp + DT;
    OMP_FOR
    for (int i = 0; i < N; i++) {
        m->rivout_a[i] = m->rivout_a[i] + m->rivout[i] * DT;
        m->fldout_a[i] = m->fldout_a[i] + m->fldout[i] * DT;
        m->rivvel_a[i] = m->rivvel_a[i] + m->rivvel[i] * DT;
        m->outflw_a[i] = m->outflw_a[i] + m->outflw[i] * DT;
        m->pthout_a[i] = (m->pthout_a[i] + m->pthout[i] * DT) - m->pthinf[i] * DT;
        m->gdwrtn_a[i] = m->gdwrtn_a[i] + m->gdwrtn[i] * DT;
        m->runoff_a[i] = m->runoff_a[i] + m->runoff[i] * DT;
        m->rofsub_a[i] = m->rofsub_a[i] + m->rofsub[i] * DT;
        m->outflw_m[i] = dmax(m->outflw_m[i], fabs(m->outflw[i]));
        m->rivdph_m[i] = dmax(m->rivdph_m[i], m->rivdph[i]);
        m->storge_m[i] = dmax(m->storge_m[i], m->storge[i]);
    }
    if (m->ldamout) for (int i = 0; i < N; i++) m->daminf_a[i] = m->daminf_a[i] + m->daminf[i] * DT;
    for (int k = 0; k < PL; k++) m->pthflw_a[k] = m->pthflw_a[k] + m->pthflw[k] * DT;
}
static void diag_getave_adpstp(orc_model *m) {
    int N = m->nseqmax, P = m->npthout;
    double n = m->nadd_adp;
    for (int i = 0; i < N; i++) {
        m->rivout_a[i] /= n; m->fldout_a[i] /= n; m->outflw_a[i] /= n; m->rivvel_a[i] /= n;
        m->pthout_a[i] /= n; m->gdwrtn_a[i] /= n; m->runoff_a[i] /= n; m->rofsub_a[i] /= n;
    }
    if (m->ldamout) for (int i = 0; i < N; i++) m->daminf_a[i] /= n;
    for (int l = 0; l < m->npthlev; l++)
        for (int p = 0; p < P; p++) {
            m->pthflw_a[(size_t)l * P + p] /= n;
            m->pthflwsum_a[p] = m->pthflwsum_a[p] + m->pthflw_a[(size_t)l * P + p];
        }
}

/* Output-interval averages and maxima, src/cmf_calc_diag_mod.F90:222-356.  CMF_DRV_ADVANCE calls
 * AVEMAX after every CMF_PHYSICS_ADVANCE (src/cmf_drv_advance_mod.F90:114), GETAVE before an output
 * write (:123) and RESET after it (:143); DT there is DT_DEF again (src/cmf_ctrl_physics_mod.F90:145). */
static void diag_reset_output(orc_model *m) {
    int N = m->nseqmax, PL = m->npthout * m->npthlev;
    m->nadd_out = 0.0;
    for (int i = 0; i < N; i++) {
        m->rivout_o[i] = m->fldout_o[i] = m->outflw_o[i] = m->rivvel_o[i] = m->pthout_o[i] = 0.0;
        m->gdwrtn_o[i] = m->runoff_o[i] = m->rofsub_o[i] = 0.0;
        m->storge_om[i] = m->outflw_om[i] = m->rivdph_om[i] = 0.0;
    }
    if (m->ldamout) for (int i = 0; i < N; i++) m->daminf_o[i] = 0.0;
    for (int k = 0; k < PL; k++) m->pthflw_o[k] = 0.0;
}
static void diag_avemax_output(orc_model *m) {
    int N = m->nseqmax, PL = m->npthout * m->npthlev;
    double DT = m->dt;
    m->nadd_out = m->nadd_out + DT;
    OMP_FOR
    for (int i = 0; i < N; i++) {
        m->rivout_o[i] = m->rivout_o[i] + m->rivout_a[i] * DT;
        m->fldout_o[i] = m->fldout_o[i] + m->fldout_a[i] * DT;
        m->rivvel_o[i] = m->rivvel_o[i] + m->rivvel_a[i] * DT;
        m->outflw_o[i] = m->outflw_o[i] + m->outflw_a[i] * DT;
        m->pthout_o[i] = m->pthout_o[i] + m->pthout_a[i] * DT;
        m->gdwrtn_o[i] = m->gdwrtn_o[i] + m->gdwrtn_a[i] * DT;
        m->runoff_o[i] = m->runoff_o[i] + m->runoff_a[i] * DT;
        m->rofsub_o[i] = m->rofsub_o[i] + m->rofsub_a[i] * DT;
        m->outflw_om[i] = dmax(m->outflw_om[i], fabs(m->outflw_m[i]));
        m->rivdph_om[i] = dmax(m->rivdph_om[i], m->rivdph_m[i]);
        m->storge_om[i] = dmax(m->storge_om[i], m->storge_m[i]);
    }
    if (m->ldamout) for (int i = 0; i < N; i++) m->daminf_o[i] = m->daminf_o[i] + m->daminf_a[i] * DT;
    for (int k = 0; k < PL; k++) m->pthflw_o[k] = m->pthflw_o[k] + m->pthflw_a[k] * DT;
}
static void diag_getave_output(orc_model *m) {
    int N = m->nseqmax, PL = m->npthout * m->npthlev;
    double n = m->nadd_out;
    for (int i = 0; i < N; i++) {
        m->rivout_o[i] /= n; m->fldout_o[i] /= n; m->outflw_o[i] /= n; m->rivvel_o[i] /= n;
        m->pthout_o[i] /= n; m->gdwrtn_o[i] /= n; m->runoff_o[i] /= n; m->rofsub_o[i] /= n;
        if (m->ldamout) m->daminf_o[i] /= n;
    }
    for (int k = 0; k < PL; k++) m->pthflw_o[k] /= n;
}
/* op 0: CMF_DIAG_RESET_OUTPUT, 1: CMF_DIAG_AVEMAX_OUTPUT, 2: CMF_DIAG_GETAVE_OUTPUT */
void orc_diag_output(orc_model *m, int op) {
    if (op == 0) diag_reset_output(m);
    else if (op == 1) diag_avemax_output(m);
    else if (op == 2) diag_getave_output(m);
}
double orc_nadd_out(const orc_model *m) { return m->nadd_out; }

/* ============================================================================ ADVANCE */
/* CMF_PHYSICS_ADVANCE, src/cmf_ctrl_physics_mod.F90:21-153, split where the reference places
 * CMF_MPI_ADPSTP (:200-202): orc_stage returns this domain's DT_MIN, orc_substeps takes the
 * (possibly all-reduced) DT_MIN and runs the NT sub-steps. */
double orc_stage(orc_model *m) {
    int N = m->nseqall, R = m->nseqriv;
    double DT_DEF = m->dt;
    physics_fldstg(m);
    double dt_min = DT_DEF;
    if (m->ladpstp) {                                  /* CALC_ADPSTP, :161-210 */
        for (int i = 0; i < R; i++) {
            if (m->i2mask[i] == 0) {
                double ddph = dmax(m->rivdph[i], 0.01), ddst = m->nxtdst[i];
                dt_min = dmin(dt_min, (m->pcadp * ddst) * opow(m->pgrv * ddph, -0.5));
            }
        }
        for (int i = R; i < N; i++) {
            if (m->i2mask[i] == 0) {
                double ddph = dmax(m->rivdph[i], 0.01), ddst = m->pdstmth;
                dt_min = dmin(dt_min, (m->pcadp * ddst) * opow(m->pgrv * ddph, -0.5));
            }
        }
    }
    return dt_min;
}

int orc_substeps(orc_model *m, double dt_min, int *nt_out, double *dt_out) {
    double DT_DEF = m->dt;
    int NT = 1;
    double DT = DT_DEF;
    if (m->ladpstp) {
        NT = (int)(DT_DEF * (1.0 / dt_min) - F(0.01)) + 1;
        DT = DT_DEF * (double)(1.0f / (float)NT);
        m->last_dtmin = dt_min;
    }
    diag_reset_adpstp(m);
    for (int it = 1; it <= NT; it++) {
        calc_outflw(m, DT);
        if (!m->lfldout) for (int i = 0; i < m->nseqmax; i++) { m->fldout[i] = 0.0; m->fldout_pre[i] = 0.0; }
        if (m->ldamout) damout_calc(m, DT);
        if (m->lpthout) { if (m->llevee) levee_opt_pthout(m, DT); else calc_pthout(m, DT); }
        calc_inflow_lspamat(m, DT);
        if (m->ldamout) damout_watbal(m, DT);
        /* CALC_VARS_PRE, :254-277 */
        for (int i = 0; i < m->nseqmax; i++) {
            m->rivout_pre[i] = m->rivout[i]; m->rivdph_pre[i] = m->rivdph[i];
            m->fldout_pre[i] = m->fldout[i]; m->fldsto_pre[i] = m->fldsto[i];
        }
        if (m->lpthout) memcpy(m->pthflw_pre, m->pthflw, sizeof(double) * (size_t)m->npthout * m->npthlev);
        calc_stonxt(m, DT);
        physics_fldstg(m);
        if (m->substep_hook) m->substep_hook(m->substep_ctx, it);
        diag_avemax_adpstp(m, DT);
    }
    diag_getave_adpstp(m);
    m->last_nt = NT; m->last_dt = DT;
    if (nt_out) *nt_out = NT;
    if (dt_out) *dt_out = DT;
    return 0;
}

/* A test hook called after each sub-step's stage update, before CMF_DIAG_AVEMAX_ADPSTP reads the
 * sub-step's fields (NULL removes it). */
void orc_set_substep_hook(orc_model *m, void (*fn)(void *, int), void *ctx) {
    m->substep_hook = fn;
    m->substep_ctx = ctx;
}

int orc_physics_advance(orc_model *m, int *nt_out, double *dt_out) {
    const double dt_min = orc_stage(m);
    return orc_substeps(m, dt_min, nt_out, dt_out);
}

/* ============================================================================ RESTART */
/* Record I of a direct-access binary restart: one NX x NY map (FP64 when LRESTDBL, else FP32),
 * cells outside the sequence hold DMIS / RMIS = 1.E20 (src/cmf_ctrl_nmlist_mod.F90:235-236).
 * vecP2mapP / vecP2mapR, src/cmf_utils_mod.F90:111-154. */
static int rest_write_map(const orc_model *m, FILE *f, const double *vec, int dbl) {
    size_t nxy = (size_t)m->nx * m->ny;
    if (dbl) {
        double *map = dalloc(nxy);
        for (size_t k = 0; k < nxy; k++) map[k] = 1.E20;
        for (int i = 0; i < m->nseqmax; i++) map[(size_t)(m->i1seqy[i] - 1) * m->nx + (m->i1seqx[i] - 1)] = vec[i];
        size_t w = fwrite(map, sizeof(double), nxy, f);
        free(map);
        return w == nxy ? 0 : -1;
    }
    float *map = (float *)calloc(nxy, sizeof(float));
    for (size_t k = 0; k < nxy; k++) map[k] = 1.E20f;
    for (int i = 0; i < m->nseqmax; i++) map[(size_t)(m->i1seqy[i] - 1) * m->nx + (m->i1seqx[i] - 1)] = (float)vec[i];
    size_t w = fwrite(map, sizeof(float), nxy, f);
    free(map);
    return w == nxy ? 0 : -1;
}

/* mapP2vecP, src/cmf_utils_mod.F90:328-345 (a FP32 record is promoted once) */
static int rest_read_map(const orc_model *m, FILE *f, double *vec, int dbl) {
    size_t nxy = (size_t)m->nx * m->ny;
    double *map = dalloc(nxy);
    if (dbl) {
        if (fread(map, sizeof(double), nxy, f) != nxy) { free(map); return -1; }
    } else {
        float *r = (float *)calloc(nxy, sizeof(float));
        if (fread(r, sizeof(float), nxy, f) != nxy) { free(r); free(map); return -1; }
        for (size_t k = 0; k < nxy; k++) map[k] = (double)r[k];
        free(r);
    }
    for (int i = 0; i < m->nseqmax; i++) vec[i] = map[(size_t)(m->i1seqy[i] - 1) * m->nx + (m->i1seqx[i] - 1)];
    free(map);
    return 0;
}

/* WRTE_REST_BIN, src/cmf_ctrl_restart_mod.F90:389-482: records rivsto, fldsto, [rivout_pre,
 * fldout_pre, rivdph_pre, fldsto_pre unless LSTOONLY], [damsto if LDAMOUT], [levsto if LLEVEE];
 * bifurcation flows in <file>.pth as one (NPTHOUT,NPTHLEV) record.  The caller names the file
 * (the reference builds CRESTDIR//CVNREST//YYYYMMDDHH//'.bin'). */
int orc_write_restart(orc_model *m, const char *file, int dbl, int stoonly) {
    FILE *f = fopen(file, "wb");
    if (!f) return -1;
    int rc = rest_write_map(m, f, m->rivsto, dbl) | rest_write_map(m, f, m->fldsto, dbl);
    if (!stoonly)
        rc |= rest_write_map(m, f, m->rivout_pre, dbl) | rest_write_map(m, f, m->fldout_pre, dbl) |
              rest_write_map(m, f, m->rivdph_pre, dbl) | rest_write_map(m, f, m->fldsto_pre, dbl);
    if (m->ldamout) rc |= rest_write_map(m, f, m->damsto, dbl);
    if (m->llevee) rc |= rest_write_map(m, f, m->levsto, dbl);
    fclose(f);
    if (rc) return -1;
    if (m->lpthout) {
        char pth[1100];
        snprintf(pth, sizeof pth, "%s.pth", file);
        FILE *g = fopen(pth, "wb");
        if (!g) return -1;
        size_t n = (size_t)m->npthout * m->npthlev, w;
        if (dbl) w = fwrite(m->pthflw_pre, sizeof(double), n, g);
        else {
            float *r = (float *)calloc(n ? n : 1, sizeof(float));
            for (size_t k = 0; k < n; k++) r[k] = (float)m->pthflw_pre[k];
            w = fwrite(r, sizeof(float), n, g);
            free(r);
        }
        fclose(g);
        if (w != n) return -1;
    }
    return 0;
}

/* CMF_RESTART_INIT + READ_REST_BIN, src/cmf_ctrl_restart_mod.F90:91-204: prognostics zeroed, the
 * records read back; D2RIVOUT/D2FLDOUT/D1PTHFLW stay zero (the binary path does not set them);
 * LSTOONLY: D2FLDSTO_PRE = P2FLDSTO (:130-132) and D1PTHFLW_PRE = 0. */
int orc_read_restart(orc_model *m, const char *file, int dbl, int stoonly) {
    int N = m->nseqmax;
    size_t PL = (size_t)m->npthout * m->npthlev;
    for (int i = 0; i < N; i++) {
        m->rivsto[i] = m->fldsto[i] = m->rivout[i] = m->fldout[i] = 0.0;
        m->rivout_pre[i] = m->fldout_pre[i] = m->rivdph_pre[i] = m->fldsto_pre[i] = 0.0;
        if (m->ldamout) m->damsto[i] = 0.0;
        if (m->llevee) m->levsto[i] = 0.0;
    }
    if (m->lpthout) for (size_t k = 0; k < PL; k++) m->pthflw[k] = m->pthflw_pre[k] = 0.0;
    FILE *f = fopen(file, "rb");
    if (!f) return -1;
    int rc = rest_read_map(m, f, m->rivsto, dbl) | rest_read_map(m, f, m->fldsto, dbl);
    if (!stoonly)
        rc |= rest_read_map(m, f, m->rivout_pre, dbl) | rest_read_map(m, f, m->fldout_pre, dbl) |
              rest_read_map(m, f, m->rivdph_pre, dbl) | rest_read_map(m, f, m->fldsto_pre, dbl);
    if (m->ldamout) rc |= rest_read_map(m, f, m->damsto, dbl);
    if (m->llevee) rc |= rest_read_map(m, f, m->levsto, dbl);
    fclose(f);
    if (rc) return -1;
    if (m->lpthout && !stoonly) {
        char pth[1100];
        snprintf(pth, sizeof pth, "%s.pth", file);
        FILE *g = fopen(pth, "rb");
        if (!g) return -1;
        size_t r;
        if (dbl) r = fread(m->pthflw_pre, sizeof(double), PL, g);
        else {
            float *v = (float *)calloc(PL ? PL : 1, sizeof(float));
            r = fread(v, sizeof(float), PL, g);
            for (size_t k = 0; k < PL; k++) m->pthflw_pre[k] = (double)v[k];
            free(v);
        }
        fclose(g);
        if (r != PL) return -1;
    }
    if (stoonly) for (int i = 0; i < N; i++) m->fldsto_pre[i] = m->fldsto[i];
    return 0;
}

/* CMF_BOUNDARY_UPDATE, src/cmf_ctrl_boundary_mod.F90:267-304: D2DWNELV = D2ELEVTN (+ D2MEANSL)
 * (+ D2SEALEV); NULL leaves a term out. */
void orc_update_boundary(orc_model *m, const double *sealev, const double *meansl) {
    for (int i = 0; i < m->nseqmax; i++) {
        double v = meansl ? m->elevtn[i] + meansl[i] : m->elevtn[i];
        if (sealev) v = v + sealev[i];
        m->dwnelv[i] = v;
    }
}

/* CMF_PHYSICS_FLDSTG (stage scheme alone), src/cmf_ctrl_physics_mod.F90:288-305 */
void orc_physics_fldstg(orc_model *m) { physics_fldstg(m); }

/* CMF_CALC_OUTPRE, src/cmf_opt_outflw_mod.F90:308-421: previous-step discharge by the diffusive
 * (Manning) wave for a storage-only restart; needs the stage scheme to have run. */
void orc_calc_outpre(orc_model *m) {
    int N = m->nseqall, R = m->nseqriv;
    const double p23 = F(2. / 3.);
    for (int i = 0; i < N; i++) {
        m->sfcelv[i] = m->rivelv[i] + m->rivdph[i];
        m->rivdph_pre[i] = m->rivdph[i];
    }
    for (int i = 0; i < R; i++) {
        int j = m->i1next[i];
        double dsfcmax = dmax(m->sfcelv[i], m->sfcelv[j]);
        double dslope = (m->sfcelv[i] - m->sfcelv[j]) * (1.0 / m->nxtdst[i]);
        double dslope_f = dmax(-0.005, dmin(0.005, dslope));
        double dflw = dsfcmax - m->rivelv[i];
        double darea = m->rivwth[i] * dflw;
        if (darea > F(1.E-5)) {
            m->rivout_pre[i] = darea * (((1.0 / m->rivman[i]) * opow(dflw, p23)) * sqrt(fabs(dslope)));
            if (dslope < 0.0) m->rivout_pre[i] = -m->rivout_pre[i];
        } else m->rivout_pre[i] = 0.0;
        double dflw_f = dmax(dsfcmax - m->elevtn[i], 0.0);
        double dare_f = m->fldsto[i] * (1.0 / m->rivlen[i]);
        dare_f = dmax(dare_f - m->flddph[i] * m->rivwth[i], 0.0);
        if (dare_f > F(1.E-5)) {
            m->fldout_pre[i] = dare_f * (((1.0 / m->pmanfld) * opow(dflw_f, p23)) * sqrt(fabs(dslope_f)));
            if (dslope_f < 0.0) m->fldout_pre[i] = -m->fldout_pre[i];
        } else m->fldout_pre[i] = 0.0;
    }
    for (int i = R; i < N; i++) {
        double dslope = (m->sfcelv[i] - m->dwnelv[i]) * (1.0 / m->pdstmth);
        double dslope_f = dmax(-0.005, dmin(0.005, dslope));
        double dflw = m->rivdph[i];
        double darea = m->rivwth[i] * dflw;
        if (darea > F(1.E-5)) {
            m->rivout_pre[i] = darea * (((1.0 / m->rivman[i]) * opow(dflw, p23)) * sqrt(fabs(dslope)));
            if (dslope < 0.0) m->rivout_pre[i] = -m->rivout_pre[i];
        } else m->rivout_pre[i] = 0.0;
        double dflw_f = dmax(m->sfcelv[i] - m->elevtn[i], 0.0);
        double dare_f = m->fldsto[i] * (1.0 / m->rivlen[i]);
        dare_f = dmax(dare_f - m->flddph[i] * m->rivwth[i], 0.0);
        if (dare_f > F(1.E-5)) {
            m->fldout_pre[i] = dare_f * (((1.0 / m->pmanfld) * opow(dflw_f, p23)) * sqrt(fabs(dslope_f)));
            if (dslope_f < 0.0) m->fldout_pre[i] = -m->fldout_pre[i];
        } else m->fldout_pre[i] = 0.0;
    }
    if (m->lpthout) {
        int P = m->npthout, Lp = m->npthlev;
        for (int p = 0; p < P; p++) {
            int u = m->pth_upst[p] - 1, d = m->pth_down[p] - 1;
            if (u < 0 || d < 0) continue;          /* path outside the domain (not in the reference's loop range) */
            double dslope = (m->sfcelv[u] - m->sfcelv[d]) * (1.0 / m->pth_dst[p]);
            for (int l = 0; l < Lp; l++) {
                double dflw = dmax(m->sfcelv[u], m->sfcelv[d]) - m->pth_elv[(size_t)l * P + p];
                dflw = dmax(dflw, 0.0);
                double *o = &m->pthflw_pre[(size_t)l * P + p];
                if (dflw > F(1.E-5)) {
                    *o = (m->pth_wth[(size_t)l * P + p] * dflw) * (((1.0 / m->pth_man[l]) * opow(dflw, p23)) * sqrt(fabs(dslope)));
                    if (dslope < 0.0) *o = -*o;
                } else *o = 0.0;
            }
        }
    }
    if (!m->lfldout) for (int i = 0; i < m->nseqmax; i++) m->fldout_pre[i] = 0.0;
}

/* ============================================================================ public API */
static void set_defaults(orc_model *m) {
    m->ladpstp = 1; m->lfplain = 1; m->lfldout = 1; m->lpthout = 0; m->ldamout = 0; m->llevee = 0;
    m->lspamat = 1; m->lstg_es = 0; m->ldamh22 = 0; m->ldamyby = 0; m->livnorm = 0; m->lmeansl = 0;
    m->dt = 24 * 60 * 60; m->pmanriv = 0.03; m->pmanfld = 0.10; m->pgrv = 9.8; m->pdstmth = 10000.0;
    m->pcadp = 0.7; m->pminslp = F(1.E-5); m->drofunit = 86400000.0;
    m->npthout = 1; m->npthlev = 1;
}

orc_model *orc_create(const char *casedir, const char *nmlfile, char *errbuf, int errlen) {
    orc_model *m = (orc_model *)calloc(1, sizeof(orc_model));
    set_defaults(m);
    int rc = read_namelist(m, casedir, nmlfile ? nmlfile : "input_cmf.nam");
    char path[1024];
    if (!rc) {
        snprintf(path, sizeof path, "%s/diminfo.txt", casedir);
        FILE *f = fopen(path, "r");
        if (!f) { snprintf(m->err, sizeof m->err, "cannot open %s", path); rc = -1; }
        else {
            char line[512]; int v[3] = {0, 0, 0};
            for (int k = 0; k < 3 && fgets(line, sizeof line, f); k++) v[k] = atoi(line);
            fclose(f);
            m->nx = v[0]; m->ny = v[1]; m->nlfp = v[2];
        }
    }
    if (!rc) {
        size_t ng = (size_t)m->nx * m->ny;
        m->nextx = ialloc(ng * 2); m->nexty = m->nextx + ng;
        if (read_i32_records(m->cnextxy, m->nextx, ng, 2)) { snprintf(m->err, sizeof m->err, "cannot read nextxy"); rc = -1; }
    }
    if (!rc) rc = calc_1d_seq(m);
    if (!rc && m->lpthout) rc = read_bifparam(m);
    if (!rc && !m->lpthout) {
        m->npthout = 1; m->npthlev = 1;
        m->pth_upst = ialloc(1); m->pth_down = ialloc(1); m->pth_dst = dalloc(1);
        m->pth_elv = dalloc(1); m->pth_wth = dalloc(1); m->pth_man = dalloc(1);
        m->i1p_outn = ialloc(m->nseqmax); m->i1p_infn = ialloc(m->nseqmax);
        m->i1p_out = ialloc(1); m->i1p_inf = ialloc(1); m->onmax = m->inmax = 1;
    }
    if (!rc) rc = topo_init(m);
    if (!rc && m->llevee) rc = levee_init(m);
    if (!rc) {
        if (!m->llevee) { m->levfrc = dalloc(m->nseqmax); m->levhgt = dalloc(m->nseqmax); }
        prog_diag_init(m);
        physics_fldstg(m);
    }
    if (!rc && m->ldamout) rc = damout_init(m);
    if (!rc && !m->ldamout) { m->i1dam = ialloc(m->nseqmax); }
    if (rc) {
        if (errbuf && errlen > 0) snprintf(errbuf, (size_t)errlen, "%s", m->err);
        free(m);   /* partial allocations leak on this error path; the oracle process is short-lived */
        return NULL;
    }
    return m;
}

void orc_free(orc_model *m) { (void)m; /* process-lifetime object: arrays freed at exit */ }

/* CONV_RESOL, src/cmf_ctrl_forcing_mod.F90:795-831: runoff map (mm/dt as JPRB) -> m3/s */
int orc_put_runoff_map(orc_model *m, const double *map) {
    for (int i = 0; i < m->nseqmax; i++) {
        double v = map[(size_t)(m->i1seqy[i] - 1) * m->nx + (m->i1seqx[i] - 1)];
        if (v != F(1.E20)) {
            m->runoff[i] = (v * m->grarea[i]) / m->drofunit;
            m->runoff[i] = dmax(m->runoff[i], 0.0);
        } else m->runoff[i] = 0.0;
    }
    return 0;
}
/* CMF_FORCING_GET's cleaning of a runoff field (src/cmf_ctrl_forcing_mod.F90:486-494): NaN -> RMIS,
 * then max(., 0). */
void orc_forcing_clean(double *grid, size_t n) {
    for (size_t k = 0; k < n; k++) {
        if (isnan(grid[k])) grid[k] = F(1.E20);
        grid[k] = dmax(grid[k], 0.0);
    }
}

/* ROFF_INTERP, src/cmf_ctrl_forcing_mod.F90:760-790: D2RUNOFF(ISEQ) = sum over the input-matrix
 * entries with IXIN > 0 (inside NXIN x NYIN) of PBUFFIN(IXIN,IYIN) * INPA / DROFUNIT, skipping
 * RMIS inputs.  inpx/inpy/inpa are [INPN][NSEQMAX] (INPX(NSEQMAX,INPN) column-major); grid is
 * PBUFFIN(NXIN,NYIN). */
int orc_roff_interp(orc_model *m, const double *grid, int nxin, int nyin, int inpn, const int *inpx, const int *inpy,
                    const double *inpa) {
    int N = m->nseqmax;
    for (int i = 0; i < N; i++) {
        double out = 0.0;
        for (int k = 0; k < inpn; k++) {
            int ix = inpx[(size_t)k * N + i], iy = inpy[(size_t)k * N + i];
            if (ix > 0) {
                if (ix > nxin || iy > nyin || iy < 1) continue;
                double v = grid[(size_t)(iy - 1) * nxin + (ix - 1)];
                if (v != F(1.E20)) out = out + (v * inpa[(size_t)k * N + i]) / m->drofunit;
            }
        }
        m->runoff[i] = out;
    }
    return 0;
}

int orc_put_runoff_vec(orc_model *m, const double *vec) {
    memcpy(m->runoff, vec, sizeof(double) * (size_t)m->nseqmax);
    return 0;
}

void orc_dims(const orc_model *m, int *out) {
    out[0] = m->nx; out[1] = m->ny; out[2] = m->nlfp; out[3] = m->nseqmax; out[4] = m->nseqall;
    out[5] = m->nseqriv; out[6] = m->npthout; out[7] = m->npthlev; out[8] = m->ndam;
    out[9] = m->upnmax; out[10] = m->last_nt;
}
void orc_budget(const orc_model *m, double *out) {
    out[0] = m->glbstopre; out[1] = m->glbstonxt; out[2] = m->glbstonew; out[3] = m->glbrivinf; out[4] = m->glbrivout;
    out[5] = m->glbstopre2; out[6] = m->glbstonew2; out[7] = m->glbrivsto; out[8] = m->glbfldsto; out[9] = m->glbfldare;
    out[10] = m->glblevsto; out[11] = m->dam_miss; out[12] = m->last_dt; out[13] = m->last_dtmin; out[14] = m->nadd_adp;
}

/* named access to every array, for the tests */
double *orc_darray(orc_model *m, const char *name, int *len) {
    int N = m->nseqmax, PL = m->npthout * m->npthlev, P = m->npthout, L = m->nlfp;
    struct { const char *n; double *p; int l; } t[] = {
        {"grarea", m->grarea, N}, {"elevtn", m->elevtn, N}, {"nxtdst", m->nxtdst, N}, {"rivlen", m->rivlen, N},
        {"rivwth", m->rivwth, N}, {"rivhgt", m->rivhgt, N}, {"fldhgt", m->fldhgt, N * L}, {"rivman", m->rivman, N},
        {"dwnelv", m->dwnelv, N}, {"rivstomax", m->rivstomax, N}, {"rivelv", m->rivelv, N},
        {"fldstomax", m->fldstomax, N * L}, {"fldgrd", m->fldgrd, N * L},
        {"levhgt", m->levhgt, m->levhgt ? N : 0}, {"levfrc", m->levfrc, m->levfrc ? N : 0},
        {"bashgt", m->bashgt, m->bashgt ? N : 0}, {"levdst", m->levdst, m->levdst ? N : 0},
        {"levbassto", m->levbassto, m->levbassto ? N : 0}, {"levtopsto", m->levtopsto, m->levtopsto ? N : 0},
        {"levfilsto", m->levfilsto, m->levfilsto ? N : 0},
        {"pth_dst", m->pth_dst, P}, {"pth_elv", m->pth_elv, PL}, {"pth_wth", m->pth_wth, PL}, {"pth_man", m->pth_man, m->npthlev},
        {"runoff", m->runoff, N}, {"rivsto", m->rivsto, N}, {"fldsto", m->fldsto, N}, {"rivout", m->rivout, N},
        {"fldout", m->fldout, N}, {"rivout_pre", m->rivout_pre, N}, {"fldout_pre", m->fldout_pre, N},
        {"rivdph_pre", m->rivdph_pre, N}, {"fldsto_pre", m->fldsto_pre, N}, {"pthflw", m->pthflw, PL},
        {"pthflw_pre", m->pthflw_pre, PL}, {"damsto", m->damsto, N}, {"daminf", m->daminf, N}, {"levsto", m->levsto, N},
        {"rivinf", m->rivinf, N}, {"rivdph", m->rivdph, N}, {"rivvel", m->rivvel, N}, {"fldinf", m->fldinf, N},
        {"flddph", m->flddph, N}, {"fldfrc", m->fldfrc, N}, {"fldare", m->fldare, N}, {"pthout", m->pthout, N},
        {"pthinf", m->pthinf, N},
        {"sfcelv", m->sfcelv, N}, {"outflw", m->outflw, N}, {"storge", m->storge, N}, {"levdph", m->levdph, N},
        {"pthflwsum", m->pthflwsum, P}, {"rate", m->rate, N}, {"stoout", m->stoout, N},
        {"rivout_aavg", m->rivout_a, N}, {"fldout_aavg", m->fldout_a, N}, {"outflw_aavg", m->outflw_a, N},
        {"rivvel_aavg", m->rivvel_a, N}, {"pthout_aavg", m->pthout_a, N}, {"runoff_aavg", m->runoff_a, N},
        {"daminf_aavg", m->daminf_a, N}, {"storge_amax", m->storge_m, N}, {"outflw_amax", m->outflw_m, N},
        {"rivdph_amax", m->rivdph_m, N}, {"pthflw_aavg", m->pthflw_a, PL}, {"pthflwsum_aavg", m->pthflwsum_a, P},
        {"rivout_oavg", m->rivout_o, N}, {"fldout_oavg", m->fldout_o, N}, {"outflw_oavg", m->outflw_o, N},
        {"rivvel_oavg", m->rivvel_o, N}, {"pthout_oavg", m->pthout_o, N}, {"runoff_oavg", m->runoff_o, N},
        {"daminf_oavg", m->daminf_o, N}, {"storge_omax", m->storge_om, N}, {"outflw_omax", m->outflw_om, N},
        {"rivdph_omax", m->rivdph_om, N}, {"pthflw_oavg", m->pthflw_o, PL},
        {"dam_fldvol", m->fldvol, m->ndam}, {"dam_convol", m->convol, m->ndam}, {"dam_emevol", m->emevol, m->ndam},
        {"dam_adjvol", m->adjvol, m->ndam}, {"dam_qn", m->qn, m->ndam}, {"dam_qf", m->qf, m->ndam}, {"dam_qa", m->qa, m->ndam},
        {"dam_norvol", m->norvol, m->ndam}, {"dam_r_volupa", m->r_volupa, m->ndam},
    };
    for (size_t k = 0; k < sizeof(t) / sizeof(t[0]); k++)
        if (!strcmp(t[k].n, name)) { if (len) *len = t[k].l; return t[k].p; }
    if (len) *len = -1;
    return NULL;
}
int *orc_iarray(orc_model *m, const char *name, int *len) {
    int N = m->nseqmax;
    struct { const char *n; int *p; int l; } t[] = {
        {"i1seqx", m->i1seqx, N}, {"i1seqy", m->i1seqy, N}, {"i1next", m->i1next, N}, {"i1upn", m->i1upn, N},
        {"i1upst", m->i1upst, N * m->upnmax}, {"i2mask", m->i2mask, N}, {"i1dam", m->i1dam, N},
        {"pth_upst", m->pth_upst, m->npthout}, {"pth_down", m->pth_down, m->npthout},
        {"i1p_outn", m->i1p_outn, N}, {"i1p_infn", m->i1p_infn, N},
        {"i1p_out", m->i1p_out, N * m->onmax}, {"i1p_inf", m->i1p_inf, N * m->inmax},
        {"damseq", m->damseq, m->ndam}, {"damstat", m->damstat, m->ndam},
    };
    for (size_t k = 0; k < sizeof(t) / sizeof(t[0]); k++)
        if (!strcmp(t[k].n, name)) { if (len) *len = t[k].l; return t[k].p; }
    if (len) *len = -1;
    return NULL;
}
int orc_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
