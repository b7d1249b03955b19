/*
 * matjes_oracle.c -- CPU restatement of the Matjes LLG / effective-field path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker); see matjes_oracle.h for the list of
 * reference routines restated here and for the pinning status.  The Hamiltonian
 * is assembled exactly like the reference assembles it: directed-pair COO
 * triplets per shell entry, combined into one sparse "MM" matrix, and the field
 * is taken by two sparse products (H m and H^T m) like ham_base mult_r/mult_l.
 * This is deliberately a different algorithm from the product's stencil kernel.
 */
#include "matjes_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <float.h>
#include <omp.h>
#endif

#define PI_D 3.14159265358979323846264338327950288

struct orc_model {
    orc_input in;
    int nmag;
    int magidx[ORC_MAXAT];   /* cell atom -> magnetic index, -1 if not magnetic */
    int magatom[ORC_MAXAT];  /* magnetic index -> cell atom */
    double pos[ORC_MAXAT][3];/* atom positions in nm */
    int64_t ncell, nsite, n3;
    /* combined MM matrix, CSR and its transpose */
    int64_t nnz;
    int64_t *rowptr, *col;
    double* val;
    int64_t *trowptr, *tcol;
    double* tval;
    /* Zeeman "BM" term: per magnetic atom coefficient mu0*muB*c_zeeman*mu_s */
    double zee[ORC_MAXAT];
    double* bfield; /* per-cell field (Tesla), 3*ncell */
    /* dipolar */
    int nrep[3];
    int64_t nk;
    double* K; /* [nk][3nmag][3nmag], K[k][r][c] = Karr(r,c,k) */
    double* KF;   /* FFT route: [9][nk] complex (re, im) transforms of K / nk, or NULL */
    int dip_direct; /* 1: the direct circular sum even where the FFT route exists */
};

static int is_pow2(int n);
static void build_dip_fft(orc_model* M);

/* ------------------------------------------------------------------ */
/* small vector helpers                                                 */
static double nrm3(const double* v) { return sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }
static void cross3(const double* a, const double* b, double* c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

void orc_input_defaults(orc_input* in) {
    memset(in, 0, sizeof(*in));
    in->c_H_J = -1.0;     /* IO-input/input_H_types.f90:85 */
    in->c_H_D = -1.0;     /* :102 */
    in->c_H_ani = 1.0;    /* :76 */
    in->c_zeeman = -1.0;  /* :80 */
    in->dip_period_cut[0] = in->dip_period_cut[1] = in->dip_period_cut[2] = 1; /* :134 */
    for (int i = 0; i < 3; i++) in->lat.L[i] = 1;
    for (int i = 0; i < 3; i++) in->lat.areal[i][i] = 1.0;
}

/* ------------------------------------------------------------------ */
/* COO accumulation                                                     */
typedef struct { int64_t r, c; double v; int64_t seq; } trip;
typedef struct { trip* t; int64_t n, cap; } tripvec;

static int tv_push(tripvec* tv, int64_t r, int64_t c, double v) {
    if (tv->n == tv->cap) {
        int64_t nc = tv->cap ? tv->cap * 2 : 1024;
        trip* nt = (trip*)realloc(tv->t, (size_t)nc * sizeof(trip));
        if (!nt) return -1;
        tv->t = nt;
        tv->cap = nc;
    }
    tv->t[tv->n].r = r;
    tv->t[tv->n].c = c;
    tv->t[tv->n].v = v;
    tv->t[tv->n].seq = tv->n;
    tv->n++;
    return 0;
}
static int cmp_rc(const void* a, const void* b) {
    const trip* x = (const trip*)a; const trip* y = (const trip*)b;
    if (x->r != y->r) return x->r < y->r ? -1 : 1;
    if (x->c != y->c) return x->c < y->c ? -1 : 1;
    return x->seq < y->seq ? -1 : (x->seq > y->seq);
}
static int cmp_cr(const void* a, const void* b) {
    const trip* x = (const trip*)a; const trip* y = (const trip*)b;
    if (x->c != y->c) return x->c < y->c ? -1 : 1;
    if (x->r != y->r) return x->r < y->r ? -1 : 1;
    return x->seq < y->seq ? -1 : (x->seq > y->seq);
}

/* get_coo (Energy/setH_util.f90:10-36): keep |h| > 1e-10*max|h|, column-major order */
typedef struct { int n; int r[9 * ORC_MAXAT * ORC_MAXAT]; int c[9 * ORC_MAXAT * ORC_MAXAT]; double v[9 * ORC_MAXAT * ORC_MAXAT]; } coo_local;
static void get_coo(const double* H, int dim, coo_local* out) {
    double maxv = 0.0;
    for (int i = 0; i < dim * dim; i++) if (fabs(H[i]) > maxv) maxv = fabs(H[i]);
    double thres = maxv * 1.0e-10;
    out->n = 0;
    for (int c = 0; c < dim; c++)
        for (int r = 0; r < dim; r++) {
            double h = H[r * dim + c];
            if (fabs(h) > thres) {
                out->r[out->n] = r; out->c[out->n] = c; out->v[out->n] = h; out->n++;
            }
        }
}

/* ------------------------------------------------------------------ */
/* neighbour shells: setup/neighbor_type.f90:78-330                     */
typedef struct { int a1, a2; int o[3]; } nb_entry;
typedef struct { double d; int64_t idx; } dsort;
static int cmp_d(const void* a, const void* b) {
    const dsort* x = (const dsort*)a; const dsort* y = (const dsort*)b;
    if (x->d != y->d) return x->d < y->d ? -1 : 1;
    return x->idx < y->idx ? -1 : (x->idx > y->idx);
}

static double min_areal_norm(const orc_lattice* L) {
    double e = 1e300;
    for (int j = 0; j < 3; j++) { double n = nrm3(L->areal[j]); if (n < e) e = n; }
    return e;
}

/* All (a1, a2, offset) entries of one requested shell rank (1 = nearest). */
static int get_shell(const orc_model* M, int t1, int t2, int rank, nb_entry** out, int* nout) {
    const orc_lattice* L = &M->in.lat;
    int id1[ORC_MAXAT], id2[ORC_MAXAT], n1 = 0, n2 = 0;
    for (int a = 0; a < L->natom; a++) {
        if (L->attype[a] == t1) id1[n1++] = a;
        if (L->attype[a] == t2) id2[n2++] = a;
    }
    if (n1 == 0 || n2 == 0) return -1;
    int nv = rank + (t1 == t2 ? 1 : 0); /* 0 distance counts as a shell for equal types */
    int ncheck = nv;
    int lo[3], hi[3];
    for (int d = 0; d < 3; d++) {
        if (L->L[d] > 1 || L->periodic[d]) { lo[d] = -ncheck; hi[d] = ncheck; }
        else { lo[d] = 0; hi[d] = 0; }
    }
    int64_t n = (int64_t)n1 * n2 * (hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1);
    dsort* ds = (dsort*)malloc((size_t)n * sizeof(dsort));
    int (*ent)[5] = malloc((size_t)n * sizeof(*ent));
    if (!ds || !ent) { free(ds); free(ent); return -2; }
    int64_t ii = 0;
    for (int i3 = lo[2]; i3 <= hi[2]; i3++)
        for (int i2 = lo[1]; i2 <= hi[1]; i2++)
            for (int i1 = lo[0]; i1 <= hi[0]; i1++)
                for (int b = 0; b < n2; b++)
                    for (int a = 0; a < n1; a++) {
                        double v[3];
                        for (int k = 0; k < 3; k++)
                            v[k] = M->pos[id2[b]][k] - M->pos[id1[a]][k] + i1 * L->areal[0][k] +
                                   i2 * L->areal[1][k] + i3 * L->areal[2][k];
                        ds[ii].d = nrm3(v);
                        ds[ii].idx = ii;
                        ent[ii][0] = id1[a]; ent[ii][1] = id2[b];
                        ent[ii][2] = i1; ent[ii][3] = i2; ent[ii][4] = i3;
                        ii++;
                    }
    qsort(ds, (size_t)n, sizeof(dsort), cmp_d);
    double eps = min_areal_norm(L) * 1.0e-7;
    /* shell starts: a new shell opens when d > (first d of the current shell) + eps */
    int64_t start_lo = -1, start_hi = n;
    int found = 0;
    double vmax = -10.0 * eps;
    for (int64_t i = 0; i < n; i++) {
        if (ds[i].d > vmax + eps) {
            found++;
            vmax = ds[i].d;
            if (found == nv) start_lo = i;
            if (found == nv + 1) { start_hi = i; break; }
        }
    }
    if (start_lo < 0) { free(ds); free(ent); return -3; }
    int cnt = (int)(start_hi - start_lo);
    nb_entry* e = (nb_entry*)malloc((size_t)cnt * sizeof(nb_entry));
    for (int k = 0; k < cnt; k++) {
        int64_t o = ds[start_lo + k].idx;
        e[k].a1 = ent[o][0]; e[k].a2 = ent[o][1];
        e[k].o[0] = ent[o][2]; e[k].o[1] = ent[o][3]; e[k].o[2] = ent[o][4];
    }
    free(ds); free(ent);
    *out = e; *nout = cnt;
    return 0;
}

/* unfold_neighbors (neighbor_type.f90:135-180): every cell pair of one entry */
typedef void (*pair_cb)(void* ctx, int64_t c1, int64_t c2);
static void unfold(const orc_lattice* L, const int o[3], pair_cb cb, void* ctx) {
    int lo[3], hi[3];
    for (int d = 0; d < 3; d++) {
        lo[d] = 1; hi[d] = L->L[d];
        if (!L->periodic[d] && o[d] < 0) lo[d] = 1 - o[d];
        if (!L->periodic[d] && o[d] > 0) hi[d] = L->L[d] - o[d];
    }
    for (int z = lo[2]; z <= hi[2]; z++)
        for (int y = lo[1]; y <= hi[1]; y++)
            for (int x = lo[0]; x <= hi[0]; x++) {
                int x2 = ((x + o[0] - 1) % L->L[0] + L->L[0]) % L->L[0];
                int y2 = ((y + o[1] - 1) % L->L[1] + L->L[1]) % L->L[1];
                int z2 = ((z + o[2] - 1) % L->L[2] + L->L[2]) % L->L[2];
                int64_t c1 = (x - 1) + (int64_t)L->L[0] * ((y - 1) + (int64_t)L->L[1] * (z - 1));
                int64_t c2 = x2 + (int64_t)L->L[0] * (y2 + (int64_t)L->L[1] * z2);
                cb(ctx, c1, c2);
            }
}

typedef struct { tripvec* tv; const coo_local* loc; int dim; int err; } add_ctx;
static void add_pair(void* vctx, int64_t c1, int64_t c2) {
    add_ctx* a = (add_ctx*)vctx;
    for (int k = 0; k < a->loc->n; k++)
        if (tv_push(a->tv, c1 * a->dim + a->loc->r[k], c2 * a->dim + a->loc->c[k], a->loc->v[k])) a->err = 1;
}

/* get_DMI (exchange_Heisenberg_D.f90:253-330): normalised sum over the mediator
 * atoms nearest to the bond centre of normalise((r_i-r_n) x (r_j-r_n)). */
static int get_dmi(const orc_model* M, const nb_entry* e, int tmed, double dmi[3]) {
    const orc_lattice* L = &M->in.lat;
    double pa[3], pb[3], cen[3];
    for (int k = 0; k < 3; k++) {
        pa[k] = M->pos[e->a1][k];
        pb[k] = M->pos[e->a2][k] + e->o[0] * L->areal[0][k] + e->o[1] * L->areal[1][k] + e->o[2] * L->areal[2][k];
        cen[k] = (pa[k] + pb[k]) * 0.5;
    }
    /* reduce the centre into the first cell with the reciprocal vectors */
    double a1[3], a2[3], a3[3];
    memcpy(a1, L->areal[0], sizeof a1); memcpy(a2, L->areal[1], sizeof a2); memcpy(a3, L->areal[2], sizeof a3);
    double c23[3], c31[3], c12[3];
    cross3(a2, a3, c23); cross3(a3, a1, c31); cross3(a1, a2, c12);
    double vol = a1[0] * c23[0] + a1[1] * c23[1] + a1[2] * c23[2];
    double fr[3] = {(cen[0] * c23[0] + cen[1] * c23[1] + cen[2] * c23[2]) / vol,
                    (cen[0] * c31[0] + cen[1] * c31[1] + cen[2] * c31[2]) / vol,
                    (cen[0] * c12[0] + cen[1] * c12[1] + cen[2] * c12[2]) / vol};
    double cuc[3];
    for (int k = 0; k < 3; k++)
        cuc[k] = cen[k] - floor(fr[0]) * L->areal[0][k] - floor(fr[1]) * L->areal[1][k] - floor(fr[2]) * L->areal[2][k];
    int lo[3], hi[3];
    for (int d = 0; d < 3; d++) {
        if (L->L[d] > 1 || L->periodic[d]) { lo[d] = -1; hi[d] = 1; } else { lo[d] = hi[d] = 0; }
    }
    double best = 1e300;
    double eps = min_areal_norm(L) * 1.0e-7;
    /* pass 1: minimal distance */
    for (int i3 = lo[2]; i3 <= hi[2]; i3++)
        for (int i2 = lo[1]; i2 <= hi[1]; i2++)
            for (int i1 = lo[0]; i1 <= hi[0]; i1++)
                for (int a = 0; a < L->natom; a++) {
                    if (L->attype[a] != tmed) continue;
                    double v[3];
                    for (int k = 0; k < 3; k++)
                        v[k] = M->pos[a][k] - cuc[k] + i1 * L->areal[0][k] + i2 * L->areal[1][k] + i3 * L->areal[2][k];
                    double d = nrm3(v);
                    if (d < best) best = d;
                }
    if (best > 1e299) return -1;
    double sum[3] = {0, 0, 0};
    for (int i3 = lo[2]; i3 <= hi[2]; i3++)
        for (int i2 = lo[1]; i2 <= hi[1]; i2++)
            for (int i1 = lo[0]; i1 <= hi[0]; i1++)
                for (int a = 0; a < L->natom; a++) {
                    if (L->attype[a] != tmed) continue;
                    double v[3], pf[3], d1[3], d2[3], cr[3];
                    for (int k = 0; k < 3; k++)
                        v[k] = M->pos[a][k] - cuc[k] + i1 * L->areal[0][k] + i2 * L->areal[1][k] + i3 * L->areal[2][k];
                    if (!(nrm3(v) <= best + eps)) continue;
                    for (int k = 0; k < 3; k++) {
                        pf[k] = M->pos[a][k] + i1 * L->areal[0][k] + i2 * L->areal[1][k] + i3 * L->areal[2][k];
                        pf[k] = pf[k] - cuc[k] + cen[k];
                        d1[k] = pa[k] - pf[k];
                        d2[k] = pb[k] - pf[k];
                    }
                    cross3(d1, d2, cr);
                    double n = nrm3(cr);
                    if (n > 1e-8) for (int k = 0; k < 3; k++) sum[k] += cr[k] / n;
                }
    double n = nrm3(sum);
    if (n > 1e-8) for (int k = 0; k < 3; k++) sum[k] /= n;
    memcpy(dmi, sum, sizeof sum);
    return 0;
}

/* ------------------------------------------------------------------ */
static int build_csr(tripvec* tv, int64_t n3, int transpose, int64_t** rp, int64_t** cl, double** vl, int64_t* nnz_out) {
    qsort(tv->t, (size_t)tv->n, sizeof(trip), transpose ? cmp_cr : cmp_rc);
    /* merge duplicates (summing in insertion order) */
    int64_t m = 0;
    for (int64_t i = 0; i < tv->n; i++) {
        int64_t r = transpose ? tv->t[i].c : tv->t[i].r;
        int64_t c = transpose ? tv->t[i].r : tv->t[i].c;
        if (m > 0) {
            int64_t pr = transpose ? tv->t[m - 1].c : tv->t[m - 1].r;
            int64_t pc = transpose ? tv->t[m - 1].r : tv->t[m - 1].c;
            if (pr == r && pc == c) { tv->t[m - 1].v += tv->t[i].v; continue; }
        }
        tv->t[m++] = tv->t[i];
    }
    int64_t* rowptr = (int64_t*)calloc((size_t)n3 + 1, sizeof(int64_t));
    int64_t* col = (int64_t*)malloc((size_t)(m ? m : 1) * sizeof(int64_t));
    double* val = (double*)malloc((size_t)(m ? m : 1) * sizeof(double));
    if (!rowptr || !col || !val) return -1;
    for (int64_t i = 0; i < m; i++) {
        int64_t r = transpose ? tv->t[i].c : tv->t[i].r;
        rowptr[r + 1]++;
        col[i] = transpose ? tv->t[i].r : tv->t[i].c;
        val[i] = tv->t[i].v;
    }
    for (int64_t r = 0; r < n3; r++) rowptr[r + 1] += rowptr[r];
    *rp = rowptr; *cl = col; *vl = val; *nnz_out = m;
    tv->n = m;
    return 0;
}

static void build_dipolar(orc_model* M) {
    const orc_lattice* L = &M->in.lat;
    int nm = M->nmag, dm = 3 * nm;
    int period[3], kb[2][3];
    /* init_shape (fft_ham_base.f90:191-220): open axes are doubled (dip_on 1);
     * dip_on 2 doubles every axis longer than one cell (linear convolution, the
     * image sums over the symmetric window of the explicit route) */
    const int full = M->in.dip_on == 2;
    for (int d = 0; d < 3; d++) {
        period[d] = L->L[d] == 1 || (L->periodic[d] && !full);
        M->nrep[d] = L->L[d];
        kb[0][d] = 0; kb[1][d] = L->L[d] - 1;
        if (!period[d]) { M->nrep[d] = 2 * L->L[d]; kb[0][d] = -L->L[d] + 1; kb[1][d] = L->L[d] - 1; }
    }
    M->nk = (int64_t)M->nrep[0] * M->nrep[1] * M->nrep[2];
    M->K = (double*)calloc((size_t)M->nk * dm * dm, sizeof(double));
    /* get_supercell_vec (dipolar_magnetic.f90:275-308) */
    int be[2][3], nr[3];
    for (int d = 0; d < 3; d++) {
        be[0][d] = be[1][d] = 0;
        if (L->periodic[d]) { be[0][d] = -M->in.dip_period_cut[d]; be[1][d] = M->in.dip_period_cut[d]; }
        nr[d] = be[1][d] - be[0][d] + 1;
    }
    int nsc = nr[0] * nr[1] * nr[2];
    double (*sc)[3] = malloc((size_t)nsc * sizeof(*sc));
    int ii = 0;
    for (int i3 = 0; i3 < nr[2]; i3++)
        for (int i2 = 0; i2 < nr[1]; i2++)
            for (int i1 = 0; i1 < nr[0]; i1++) {
                for (int k = 0; k < 3; k++)
                    sc[ii][k] = L->areal[0][k] * L->L[0] * (double)(be[0][0] + i1) +
                                L->areal[1][k] * L->L[1] * (double)(be[0][1] + i2) +
                                L->areal[2][k] * L->L[2] * (double)(be[0][2] + i3);
                ii++;
            }
    for (int i3 = kb[0][2]; i3 <= kb[1][2]; i3++) {
        int m3 = ((i3 % M->nrep[2]) + M->nrep[2]) % M->nrep[2];
        for (int i2 = kb[0][1]; i2 <= kb[1][1]; i2++) {
            int m2 = ((i2 % M->nrep[1]) + M->nrep[1]) % M->nrep[1];
            for (int i1 = kb[0][0]; i1 <= kb[1][0]; i1++) {
                int m1 = ((i1 % M->nrep[0]) + M->nrep[0]) % M->nrep[0];
                int64_t ik = m1 + (int64_t)M->nrep[0] * (m2 + (int64_t)M->nrep[1] * m3);
                double pb[3];
                for (int k = 0; k < 3; k++) pb[k] = i1 * L->areal[0][k] + i2 * L->areal[1][k] + i3 * L->areal[2][k];
                for (int ia = 0; ia < nm; ia++)
                    for (int ja = 0; ja < nm; ja++) {
                        double db[3];
                        for (int k = 0; k < 3; k++) db[k] = pb[k] + M->pos[M->magatom[ia]][k] - M->pos[M->magatom[ja]][k];
                        for (int s = 0; s < nsc; s++) {
                            double df[3] = {db[0] + sc[s][0], db[1] + sc[s][1], db[2] + sc[s][2]};
                            double r = nrm3(df);
                            if (r == 0.0) continue; /* self term vanishes (complex-eps trick, :148,158) */
                            double u[3] = {df[0] / r, df[1] / r, df[2] / r};
                            double r3 = r * r * r;
                            for (int a = 0; a < 3; a++)
                                for (int b = 0; b < 3; b++) {
                                    double t = 3.0 * u[a] * u[b] - (a == b ? 1.0 : 0.0);
                                    M->K[(ik * dm + 3 * ia + a) * dm + 3 * ja + b] += t / r3;
                                }
                        }
                    }
            }
        }
    }
    free(sc);
    for (int64_t k = 0; k < M->nk; k++)
        for (int r = 0; r < dm; r++)
            for (int c = 0; c < dm; c++) {
                double mu = L->moment[M->magatom[r / 3]] * L->moment[M->magatom[c / 3]];
                double v = M->K[(k * dm + r) * dm + c] * mu;
                M->K[(k * dm + r) * dm + c] = -v * ORC_DIP_PREF * 0.5 * 0.25 / PI_D;
            }
}

int orc_model_build(const orc_input* in, orc_model** out) {
    orc_model* M = (orc_model*)calloc(1, sizeof(orc_model));
    if (!M) return -1;
    M->in = *in;
    const orc_lattice* L = &M->in.lat;
    M->nmag = 0;
    for (int a = 0; a < L->natom; a++) {
        for (int k = 0; k < 3; k++)
            M->pos[a][k] = L->frac[a][0] * L->areal[0][k] + L->frac[a][1] * L->areal[1][k] + L->frac[a][2] * L->areal[2][k];
        if (L->moment[a] > 0.0) { M->magidx[a] = M->nmag; M->magatom[M->nmag] = a; M->nmag++; }
        else M->magidx[a] = -1;
    }
    if (M->nmag == 0) { free(M); return -2; }
    M->ncell = (int64_t)L->L[0] * L->L[1] * L->L[2];
    M->nsite = M->ncell * M->nmag;
    M->n3 = 3 * M->nsite;
    int dim = 3 * M->nmag;
    tripvec tv = {0};
    double* Ht = (double*)malloc(sizeof(double) * dim * dim);
    coo_local loc;
    int rc = 0;
    /* exchange J: exchange_Heisenberg_J.f90:78-124 */
    for (int t = 0; t < in->nJ && !rc; t++) {
        nb_entry* e; int ne;
        if (get_shell(M, in->J[t].t1, in->J[t].t2, in->J[t].shell, &e, &ne)) { rc = -3; break; }
        for (int s = 0; s < ne; s++) {
            int m1 = M->magidx[e[s].a1], m2 = M->magidx[e[s].a2];
            if (m1 < 0 || m2 < 0) continue;
            memset(Ht, 0, sizeof(double) * dim * dim);
            for (int k = 0; k < 3; k++) Ht[(3 * m1 + k) * dim + 3 * m2 + k] = in->J[t].J;
            for (int k = 0; k < dim * dim; k++) Ht[k] = in->c_H_J * Ht[k];
            get_coo(Ht, dim, &loc);
            add_ctx ac = {&tv, &loc, dim, 0};
            unfold(L, e[s].o, add_pair, &ac);
            if (ac.err) rc = -1;
        }
        free(e);
    }
    /* DMI: exchange_Heisenberg_D.f90:79-132 */
    for (int t = 0; t < in->nD && !rc; t++) {
        nb_entry* e; int ne;
        if (get_shell(M, in->D[t].t1, in->D[t].t2, in->D[t].shell, &e, &ne)) { rc = -3; break; }
        int any = 0;
        for (int s = 0; s < ne; s++) {
            double d[3];
            if (get_dmi(M, &e[s], in->D[t].tmed, d)) { rc = -4; break; }
            if (nrm3(d) <= 1e-8) continue;
            int m1 = M->magidx[e[s].a1], m2 = M->magidx[e[s].a2];
            if (m1 < 0 || m2 < 0) continue;
            any = 1;
            double Hm = in->D[t].D;
            int o1 = 3 * m1, o2 = 3 * m2;
            memset(Ht, 0, sizeof(double) * dim * dim);
            Ht[(o1 + 0) * dim + o2 + 1] = d[2] * Hm;
            Ht[(o1 + 2) * dim + o2 + 0] = d[1] * Hm;
            Ht[(o1 + 1) * dim + o2 + 2] = d[0] * Hm;
            Ht[(o1 + 1) * dim + o2 + 0] = -d[2] * Hm;
            Ht[(o1 + 0) * dim + o2 + 2] = -d[1] * Hm;
            Ht[(o1 + 2) * dim + o2 + 1] = -d[0] * Hm;
            for (int k = 0; k < dim * dim; k++) Ht[k] = in->c_H_D * Ht[k];
            get_coo(Ht, dim, &loc);
            add_ctx ac = {&tv, &loc, dim, 0};
            unfold(L, e[s].o, add_pair, &ac);
            if (ac.err) rc = -1;
        }
        free(e);
        if (!rc && !any) rc = -5; /* the reference stops: "DID NOT FIND A SINGLE DMI CONTRIBUTION" */
    }
    /* anisotropy: anisotropy_heisenberg.f90:148-201, 243-292 */
    if (!rc && in->nK > 0) {
        memset(Ht, 0, sizeof(double) * dim * dim);
        for (int t = 0; t < in->nK; t++) {
            double n = nrm3(in->K[t].axis);
            double dir[3] = {in->K[t].axis[0] / n, in->K[t].axis[1] / n, in->K[t].axis[2] / n};
            for (int a = 0; a < L->natom; a++) {
                if (L->attype[a] != in->K[t].type || M->magidx[a] < 0) continue;
                int o = 3 * M->magidx[a];
                for (int i1 = 0; i1 < 3; i1++)
                    for (int i2 = 0; i2 < 3; i2++)
                        Ht[(o + i1) * dim + o + i2] = Ht[(o + i1) * dim + o + i2] + in->K[t].K * dir[i1] * dir[i2];
            }
        }
        for (int k = 0; k < dim * dim; k++) Ht[k] = Ht[k] * in->c_H_ani;
        get_coo(Ht, dim, &loc);
        for (int64_t c = 0; c < M->ncell; c++)
            for (int k = 0; k < loc.n; k++)
                if (tv_push(&tv, c * dim + loc.r[k], c * dim + loc.c[k], loc.v[k])) rc = -1;
    }
    free(Ht);
    if (rc) { free(tv.t); free(M); return rc; }
    /* combined MM term as CSR and as its transpose */
    tripvec tv2 = {0};
    tv2.t = (trip*)malloc((size_t)(tv.n ? tv.n : 1) * sizeof(trip));
    memcpy(tv2.t, tv.t, (size_t)tv.n * sizeof(trip));
    tv2.n = tv2.cap = tv.n;
    int64_t nnz1, nnz2;
    if (build_csr(&tv, M->n3, 0, &M->rowptr, &M->col, &M->val, &nnz1) ||
        build_csr(&tv2, M->n3, 1, &M->trowptr, &M->tcol, &M->tval, &nnz2)) {
        free(tv.t); free(tv2.t); free(M); return -1;
    }
    M->nnz = nnz1;
    free(tv.t); free(tv2.t);
    /* Zeeman: zeeman.f90:64-80 */
    for (int a = 0; a < M->nmag; a++) M->zee[a] = (1.0 * ORC_MUB * in->c_zeeman) * L->moment[M->magatom[a]];
    M->in.zeeman_on = in->zeeman_on || nrm3(in->B_ext) >= 1e-8;
    M->bfield = (double*)malloc(sizeof(double) * 3 * M->ncell);
    for (int64_t c = 0; c < M->ncell; c++)
        for (int k = 0; k < 3; k++) M->bfield[3 * c + k] = in->B_ext[k];
    if (in->dip_on) {
        build_dipolar(M);
        if (M->nmag == 1 && is_pow2(M->nrep[0]) && is_pow2(M->nrep[1]) && is_pow2(M->nrep[2])) build_dip_fft(M);
    }
    *out = M;
    return 0;
}

void orc_model_free(orc_model* M) {
    if (!M) return;
    free(M->rowptr); free(M->col); free(M->val);
    free(M->trowptr); free(M->tcol); free(M->tval);
    free(M->bfield); free(M->K); free(M->KF);
    free(M);
}

int64_t orc_nsites(const orc_model* M) { return M->nsite; }
int orc_nmag(const orc_model* M) { return M->nmag; }
int64_t orc_mm_nnz(const orc_model* M) { return M->nnz; }
void orc_dip_nrep(const orc_model* M, int nrep[3]) {
    for (int d = 0; d < 3; d++) nrep[d] = M->in.dip_on ? M->nrep[d] : 0;
}

int orc_mm_coo(const orc_model* M, int64_t cap, int64_t* rows, int64_t* cols, double* vals) {
    if (cap < M->nnz) return -1;
    int64_t k = 0;
    for (int64_t r = 0; r < M->n3; r++)
        for (int64_t j = M->rowptr[r]; j < M->rowptr[r + 1]; j++) {
            rows[k] = r; cols[k] = M->col[j]; vals[k] = M->val[j]; k++;
        }
    return 0;
}

int orc_set_bfield(orc_model* M, const double* b) {
    for (int64_t c = 0; c < M->ncell; c++)
        for (int k = 0; k < 3; k++) M->bfield[3 * c + k] = b ? b[3 * c + k] : M->in.B_ext[k];
    if (b) M->in.zeeman_on = 1;
    return 0;
}

/* ------------------------------------------------------------------ */
/* FFT route of the dipolar convolution on power-of-two grids (one magnetic
 * atom per cell): our own iterative radix-2 transform (bit reversal, then
 * butterflies with twiddles from long-double sin/cos), applied along each axis
 * of the N_rep grid; H = IFFT(sum_j K_F(j,i) M_F(j)) with K_F = FFT(K)/prod(N_rep)
 * (fft_ham_fftw.f90:134-178,239-262).  Complex numbers as (re, im) pairs. */
static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

static void fft_line(double* a, int n, const double* w) {
    for (int i = 1, j = 0; i < n; i++) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            double t0 = a[2 * i], t1 = a[2 * i + 1];
            a[2 * i] = a[2 * j]; a[2 * i + 1] = a[2 * j + 1];
            a[2 * j] = t0; a[2 * j + 1] = t1;
        }
    }
    for (int len = 2; len <= n; len <<= 1) {
        int half = len >> 1, step = n / len;
        for (int i = 0; i < n; i += len)
            for (int k = 0; k < half; k++) {
                const double* wk = w + 2 * (k * step);
                double* u = a + 2 * (i + k);
                double* v = a + 2 * (i + k + half);
                double vr = v[0] * wk[0] - v[1] * wk[1], vi = v[0] * wk[1] + v[1] * wk[0];
                v[0] = u[0] - vr; v[1] = u[1] - vi;
                u[0] = u[0] + vr; u[1] = u[1] + vi;
            }
    }
}

/* in-place transform of g (x fastest, n[0] x n[1] x n[2] complex), sign -1 forward, +1 inverse */
static void fft3(double* g, const int n[3], int sign) {
    const int64_t tot = (int64_t)n[0] * n[1] * n[2];
    for (int ax = 0; ax < 3; ax++) {
        const int len = n[ax];
        if (len == 1) continue;
        double* w = (double*)malloc(sizeof(double) * len);
        const long double two_pi = 6.283185307179586476925286766559005768L;
        for (int k = 0; k < len / 2; k++) {
            long double a = two_pi * (long double)k / (long double)len;
            w[2 * k] = (double)cosl(a);
            w[2 * k + 1] = (double)(sign * sinl(a));
        }
        const int64_t stride = ax == 0 ? 1 : (ax == 1 ? n[0] : (int64_t)n[0] * n[1]);
        const int64_t nlines = tot / len;
#pragma omp parallel
        {
            double* line = (double*)malloc(sizeof(double) * 2 * len);
#pragma omp for schedule(static)
            for (int64_t l = 0; l < nlines; l++) {
                /* line l: all points sharing the other two coordinates */
                const int64_t lo = l % stride, hi = l / stride;
                const int64_t base = lo + hi * stride * len;
                for (int q = 0; q < len; q++) {
                    line[2 * q] = g[2 * (base + q * stride)];
                    line[2 * q + 1] = g[2 * (base + q * stride) + 1];
                }
                fft_line(line, len, w);
                for (int q = 0; q < len; q++) {
                    g[2 * (base + q * stride)] = line[2 * q];
                    g[2 * (base + q * stride) + 1] = line[2 * q + 1];
                }
            }
            free(line);
        }
        free(w);
    }
}

/* K_F of the nine components, scaled by 1/prod(N_rep) (once per model) */
static void build_dip_fft(orc_model* M) {
    const int64_t nk = M->nk;
    M->KF = (double*)malloc(sizeof(double) * 2 * 9 * nk);
    for (int c = 0; c < 9; c++) {
        double* g = M->KF + 2 * c * nk;
        for (int64_t k = 0; k < nk; k++) { g[2 * k] = M->K[k * 9 + c]; g[2 * k + 1] = 0.0; }
        fft3(g, M->nrep, -1);
        for (int64_t k = 0; k < 2 * nk; k++) g[k] = g[k] / (double)nk;
    }
}

static void dip_H_fft(const orc_model* M, const double* m, double* H) {
    const orc_lattice* L = &M->in.lat;
    const int64_t nk = M->nk;
    const int* nr = M->nrep;
    double* g = (double*)calloc((size_t)(2 * 3 * nk), sizeof(double));
    for (int64_t x = 0; x < M->ncell; x++) {
        int64_t xx = x % L->L[0], xy = (x / L->L[0]) % L->L[1], xz = x / ((int64_t)L->L[0] * L->L[1]);
        int64_t q = xx + (int64_t)nr[0] * (xy + (int64_t)nr[1] * xz);
        for (int c = 0; c < 3; c++) g[2 * (c * nk + q)] = m[3 * x + c];
    }
    for (int c = 0; c < 3; c++) fft3(g + 2 * c * nk, nr, -1);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < nk; k++) {
        double mr[3], mi[3], hr[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
        for (int j = 0; j < 3; j++) { mr[j] = g[2 * (j * nk + k)]; mi[j] = g[2 * (j * nk + k) + 1]; }
        /* H_F(i) = sum_j K_F(j,i) M_F(j)  (fft_ham_fftw.f90:249-253) */
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) {
                const double* kf = M->KF + 2 * ((j * 3 + i) * nk + k);
                hr[i] += kf[0] * mr[j] - kf[1] * mi[j];
                hi[i] += kf[0] * mi[j] + kf[1] * mr[j];
            }
        for (int i = 0; i < 3; i++) { g[2 * (i * nk + k)] = hr[i]; g[2 * (i * nk + k) + 1] = hi[i]; }
    }
    for (int c = 0; c < 3; c++) fft3(g + 2 * c * nk, nr, +1);
    for (int64_t x = 0; x < M->ncell; x++) {
        int64_t xx = x % L->L[0], xy = (x / L->L[0]) % L->L[1], xz = x / ((int64_t)L->L[0] * L->L[1]);
        int64_t q = xx + (int64_t)nr[0] * (xy + (int64_t)nr[1] * xz);
        for (int c = 0; c < 3; c++) H[3 * x + c] = g[2 * (c * nk + q)];
    }
    free(g);
}

/* dipolar field H = K * M as the direct circular convolution over the
 * N_rep grid (identical in exact arithmetic to the FFT route of
 * fft_ham_fftw.f90:239-262 with the 1/prod(N_rep) normalised K_F); the FFT
 * route above replaces it on power-of-two grids unless dip_direct is set. */
static void dip_H_direct(const orc_model* M, const double* m, double* H);
static void dip_H(const orc_model* M, const double* m, double* H) {
    if (M->KF && !M->dip_direct) dip_H_fft(M, m, H);
    else dip_H_direct(M, m, H);
}
void orc_dip_direct(orc_model* M, int direct) { M->dip_direct = direct; }

static void dip_H_direct(const orc_model* M, const double* m, double* H) {
    const orc_lattice* L = &M->in.lat;
    int nm = M->nmag, dm = 3 * nm;
    int64_t nc = M->ncell;
#pragma omp parallel for schedule(static)
    for (int64_t x = 0; x < nc; x++) {
        int xx = (int)(x % L->L[0]), xy = (int)((x / L->L[0]) % L->L[1]), xz = (int)(x / ((int64_t)L->L[0] * L->L[1]));
        double acc[3 * ORC_MAXAT];
        for (int i = 0; i < dm; i++) acc[i] = 0.0;
        for (int64_t y = 0; y < nc; y++) {
            int yx = (int)(y % L->L[0]), yy = (int)((y / L->L[0]) % L->L[1]), yz = (int)(y / ((int64_t)L->L[0] * L->L[1]));
            int d1 = ((xx - yx) % M->nrep[0] + M->nrep[0]) % M->nrep[0];
            int d2 = ((xy - yy) % M->nrep[1] + M->nrep[1]) % M->nrep[1];
            int d3 = ((xz - yz) % M->nrep[2] + M->nrep[2]) % M->nrep[2];
            const double* Kk = M->K + ((d1 + (int64_t)M->nrep[0] * (d2 + (int64_t)M->nrep[1] * d3)) * dm) * dm;
            const double* my = m + y * dm;
            /* H_F(i) = sum_j K_F(j,i) M_F(j)  (fft_ham_fftw.f90:249-253) */
            for (int i = 0; i < dm; i++) {
                double s = 0.0;
                for (int j = 0; j < dm; j++) s += Kk[j * dm + i] * my[j];
                acc[i] += s;
            }
        }
        for (int i = 0; i < dm; i++) H[x * dm + i] = acc[i];
    }
}

static void field_impl(const orc_model* M, const double* m, double* B, double* e_site,
                       double* B_mm, double* B_zee, double* B_dip, double* Etot) {
    int nm = M->nmag;
    int64_t n3 = M->n3;
    double* Hd = NULL;
    if (M->in.dip_on) {
        Hd = (double*)malloc(sizeof(double) * n3);
        dip_H(M, m, Hd);
    }
    double e_mm = 0.0, e_z = 0.0, e_d = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : e_mm, e_z, e_d)
    for (int64_t s = 0; s < M->nsite; s++) {
        double es = 0.0;
        int64_t cell = s / nm;
        int a = (int)(s % nm);
        for (int k = 0; k < 3; k++) {
            int64_t r = 3 * s + k;
            double hm = 0.0, htm = 0.0;
            for (int64_t j = M->rowptr[r]; j < M->rowptr[r + 1]; j++) hm += M->val[j] * m[M->col[j]];
            for (int64_t j = M->trowptr[r]; j < M->trowptr[r + 1]; j++) htm += M->tval[j] * m[M->tcol[j]];
            double acc = hm;            /* B += H m   (mult_r, alpha=beta=1) */
            acc = htm + acc;            /* B += H^T m (mult_l) */
            double bz = 0.0;
            if (M->in.zeeman_on) bz = M->zee[a] * M->bfield[3 * cell + k];
            double b = bz + acc;        /* B += Hz^T b */
            b = -b;                     /* field is the negative derivative */
            double hd = Hd ? Hd[r] : 0.0;
            if (Hd) b = b - 2.0 * hd;
            if (B) B[r] = b;
            if (B_mm) B_mm[r] = -(htm + hm);
            if (B_zee) B_zee[r] = -bz;
            if (B_dip) B_dip[r] = Hd ? -2.0 * hd : 0.0;
            double em = m[r] * hm;
            double ez = M->in.zeeman_on ? M->bfield[3 * cell + k] * (M->zee[a] * m[r]) : 0.0;
            double ed = Hd ? m[r] * hd : 0.0;
            e_mm += em; e_z += ez; e_d += ed;
            es += em + ez + 2.0 * ed;
        }
        if (e_site) e_site[s] = es;
    }
    if (Etot) *Etot = e_mm + e_z + e_d;
    free(Hd);
}

void orc_field(const orc_model* M, const double* m, double* B, double* e_site) {
    field_impl(M, m, B, e_site, NULL, NULL, NULL, NULL);
}
void orc_field_terms(const orc_model* M, const double* m, double* Bm, double* Bz, double* Bd) {
    field_impl(M, m, NULL, NULL, Bm, Bz, Bd, NULL);
}
double orc_energy(const orc_model* M, const double* m) {
    double E = 0.0;
    /* deterministic (serial) total: H%energy = sum over terms of m_l^T H m_r */
    int nm = M->nmag;
    double* Hd = NULL;
    if (M->in.dip_on) { Hd = (double*)malloc(sizeof(double) * M->n3); dip_H(M, m, Hd); }
    double e_mm = 0.0, e_z = 0.0, e_d = 0.0;
    for (int64_t r = 0; r < M->n3; r++) {
        double hm = 0.0;
        for (int64_t j = M->rowptr[r]; j < M->rowptr[r + 1]; j++) hm += M->val[j] * m[M->col[j]];
        e_mm += m[r] * hm;
        int64_t s = r / 3; int k = (int)(r % 3);
        if (M->in.zeeman_on) e_z += M->bfield[3 * (s / nm) + k] * (M->zee[s % nm] * m[r]);
        if (Hd) e_d += Hd[r] * m[r];
    }
    free(Hd);
    E = e_mm + e_z + e_d;
    return E;
}

/* explicit O(N^2) dipolar (dipolar_magnetic.f90:181-273), field = -(H+H^T) m */
void orc_dipolar_explicit_field(const orc_model* M, const double* m, double* B) {
    const orc_lattice* L = &M->in.lat;
    int nm = M->nmag;
    int be[2][3], nr[3];
    for (int d = 0; d < 3; d++) {
        be[0][d] = be[1][d] = 0;
        if (L->periodic[d]) { be[0][d] = -M->in.dip_period_cut[d]; be[1][d] = M->in.dip_period_cut[d]; }
        nr[d] = be[1][d] - be[0][d] + 1;
    }
    int nsc = nr[0] * nr[1] * nr[2];
    double (*sc)[3] = malloc((size_t)nsc * sizeof(*sc));
    int ii = 0;
    for (int i3 = 0; i3 < nr[2]; i3++)
        for (int i2 = 0; i2 < nr[1]; i2++)
            for (int i1 = 0; i1 < nr[0]; i1++) {
                for (int k = 0; k < 3; k++)
                    sc[ii][k] = L->areal[0][k] * L->L[0] * (double)(be[0][0] + i1) +
                                L->areal[1][k] * L->L[1] * (double)(be[0][1] + i2) +
                                L->areal[2][k] * L->L[2] * (double)(be[0][2] + i3);
                ii++;
            }
    int64_t N = M->nsite;
    double pref = -ORC_DIP_PREF * 0.5 * 0.25 / PI_D;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; i++) {
        int64_t ci = i / nm; int ai = (int)(i % nm);
        double pi[3];
        int xi = (int)(ci % L->L[0]), yi = (int)((ci / L->L[0]) % L->L[1]), zi = (int)(ci / ((int64_t)L->L[0] * L->L[1]));
        for (int k = 0; k < 3; k++) pi[k] = xi * L->areal[0][k] + yi * L->areal[1][k] + zi * L->areal[2][k] + M->pos[M->magatom[ai]][k];
        double acc[3] = {0, 0, 0};
        for (int64_t j = 0; j < N; j++) {
            int64_t cj = j / nm; int aj = (int)(j % nm);
            int xj = (int)(cj % L->L[0]), yj = (int)((cj / L->L[0]) % L->L[1]), zj = (int)(cj / ((int64_t)L->L[0] * L->L[1]));
            double pj[3];
            for (int k = 0; k < 3; k++) pj[k] = xj * L->areal[0][k] + yj * L->areal[1][k] + zj * L->areal[2][k] + M->pos[M->magatom[aj]][k];
            double T[9] = {0};
            for (int s = 0; s < nsc; s++) {
                double df[3] = {pj[0] - pi[0] + sc[s][0], pj[1] - pi[1] + sc[s][1], pj[2] - pi[2] + sc[s][2]};
                double r = nrm3(df);
                if (r == 0.0) continue;
                double u[3] = {df[0] / r, df[1] / r, df[2] / r};
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++)
                        T[a * 3 + b] += (3.0 * u[a] * u[b] - (a == b)) / (r * r * r) *
                                        L->moment[M->magatom[aj]] * L->moment[M->magatom[ai]];
            }
            /* H_ij = pref*T (symmetric in (i,j) and in (a,b)): (H + H^T) m = 2 H m */
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) acc[a] += 2.0 * pref * T[a * 3 + b] * m[3 * j + b];
        }
        for (int a = 0; a < 3; a++) B[3 * i + a] = -acc[a];
    }
    free(sc);
}

/* ------------------------------------------------------------------ */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), counter-based.    */
static void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    for (int r = 0; r < 10; r++) {
        if (r > 0) { k0 += W0; k1 += W1; }
        uint64_t p0 = (uint64_t)M0 * c[0];
        uint64_t p1 = (uint64_t)M1 * c[2];
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
    }
}
/* Box-Muller with table-driven FP64 log and sin/cos (the same evaluation as the
 * product's: every step one rounded operation or an explicit fma, no contraction):
 *   tab[2i], tab[2i+1]         (sin, cos)(2 pi (i + 1/2)/1024), i = 0..1023
 *   tab[2048+2j], tab[2049+2j] (1/F_j, ln F_j), F_j = 1 + (j + 1/2)/1024
 *   ln u = e ln2 + ln F + ln(1 + r), u = 2^e m, m in [1, 2), j = the top ten
 *   mantissa bits, r = m/F - 1, ln(1 + r) to r^4;
 *   sin/cos(a_i + x) for 2 pi (w + 1/2) 2^-32, i = w >> 22, |x| <= pi/1024,
 *   sin x to x^5, cos x - 1 to x^4.
 * One Philox block per site and step, counter (site, step, stream, 0):
 *   (r1 cos t1, r1 sin t1, r2 cos t2), r = sqrt(-2 ln u), u = (w0 + 1/2) 2^-32,
 *   (w2 + 1/2) 2^-32, t = 2 pi (w + 1/2) 2^-32 for w1, w3. */
static double g_tab[4096];
static int g_tab_ready = 0;
#define LN2_D 0.6931471805599453
#define TWO_PI_OVER_2P32 1.4629180792671596e-09
#define PI_OVER_2P32 7.314590396335798e-10

static void noise_tables(void) {
    if (g_tab_ready) return;
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (int i = 0; i < 1024; i++) {
        long double a = two_pi * ((long double)i + 0.5L) / 1024.0L;
        g_tab[2 * i] = (double)sinl(a);
        g_tab[2 * i + 1] = (double)cosl(a);
    }
    for (int j = 0; j < 1024; j++) {
        long double F = 1.0L + ((long double)j + 0.5L) / 1024.0L;
        g_tab[2048 + 2 * j] = (double)(1.0L / F);
        g_tab[2048 + 2 * j + 1] = (double)logl(F);
    }
    g_tab_ready = 1;
}

/* u = (w + 1/2) 2^-32, exact */
static double u32_half(uint32_t w) { return fma((double)w, 0x1p-32, 0x1p-33); }

static double tab_log(double u) {
    uint64_t b;
    memcpy(&b, &u, 8);
    int e = (int)((b >> 52) & 0x7ff) - 1023;
    int j = (int)((b >> 42) & 0x3ff);
    uint64_t mb = (b & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL;
    double m;
    memcpy(&m, &mb, 8);
    double r = fma(m, g_tab[2048 + 2 * j], -1.0);
    double p = fma(fma(r, -0.25, 1.0 / 3.0), r, -0.5);
    double l1p = fma(r * r, p, r);
    return fma((double)e, LN2_D, g_tab[2048 + 2 * j + 1] + l1p);
}

static void sincos2pi_word(uint32_t w, double* s, double* c) {
    int i = (int)(w >> 22);
    int d = (int)(w & 0x3fffffu) - 2097152;
    double x = fma((double)d, TWO_PI_OVER_2P32, PI_OVER_2P32);
    double x2 = x * x;
    double sx = fma(x * x2, fma(x2, 1.0 / 120.0, -1.0 / 6.0), x);
    double cm = x2 * fma(x2, 1.0 / 24.0, -0.5);
    double S = g_tab[2 * i], Cc = g_tab[2 * i + 1];
    *s = S + fma(S, cm, Cc * sx);
    *c = Cc + fma(Cc, cm, -(S * sx));
}

static void philox_site(uint64_t seed, uint32_t step, uint32_t stream, uint32_t site, double out[3]) {
    uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    uint32_t c[4] = {site, step, stream, 0u};
    philox4x32_10(c, k0, k1);
    double r1 = sqrt(-2.0 * tab_log(u32_half(c[0])));
    double r2 = sqrt(-2.0 * tab_log(u32_half(c[2])));
    double s1, c1, s2, c2;
    sincos2pi_word(c[1], &s1, &c1);
    sincos2pi_word(c[3], &s2, &c2);
    (void)s2;
    out[0] = r1 * c1;
    out[1] = r1 * s1;
    out[2] = r2 * c2;
}

void orc_tab_eval(const uint32_t* w, int64_t n, double* lg, double* s, double* c) {
    noise_tables();
    for (int64_t i = 0; i < n; i++) {
        lg[i] = tab_log(u32_half(w[i]));
        sincos2pi_word(w[i], s + i, c + i);
    }
}

void orc_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
    philox4x32_10(c, key[0], key[1]);
    memcpy(out, c, sizeof c);
}
void orc_philox_normals(uint64_t seed, uint32_t step, uint32_t stream, int64_t site0, int64_t n, double* out) {
    noise_tables();
    for (int64_t i = 0; i < n; i++) philox_site(seed, step, stream, (uint32_t)(site0 + i), out + 3 * i);
}

/* ------------------------------------------------------------------ */
/* LLG (propagator.f90:13-58): D = -[m^ x B + a m^ x (m^ x B)]/(1+a^2)  */
void orc_llg_torque(const double* B, double alpha, const double* m, double* D, int64_t n) {
    double den = 1.0 + alpha * alpha;
    for (int64_t i = 0; i < n; i++) {
        const double* mi = m + 3 * i; const double* b = B + 3 * i;
        double nr = nrm3(mi);
        double mn[3] = {mi[0], mi[1], mi[2]};
        if (nr > 1e-8) for (int k = 0; k < 3; k++) mn[k] = mi[k] / nr;
        double t[3], l[3], o[3];
        cross3(mn, b, t);
        for (int k = 0; k < 3; k++) l[k] = b[k] + alpha * t[k];
        cross3(mn, l, o);
        for (int k = 0; k < 3; k++) D[3 * i + k] = -o[k] / den;
    }
}

/* euler (solver.f90:97-118): t = m + Dint dt/hbar + DT dt/hbar, projected to |m| */
static void euler_update(const double* m, const double* Dint, const double* DT, double dt, double* out, int64_t n) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) {
        const double* mi = m + 3 * i;
        double t[3];
        for (int k = 0; k < 3; k++) {
            t[k] = mi[k] + Dint[3 * i + k] * dt / ORC_HBAR;
            if (DT) t[k] = t[k] + DT[3 * i + k] * dt / ORC_HBAR;
        }
        double nm = nrm3(mi), nt = nrm3(t);
        if (nt > 1e-8) for (int k = 0; k < 3; k++) out[3 * i + k] = t[k] * nm / nt;
        else for (int k = 0; k < 3; k++) out[3 * i + k] = mi[k];
    }
}

/* SIB stage (Mentink et al. 2010): y = m + ((m + y)/2) x a, a = dt*Omega(p, B+b),
 * Omega = -(H + alpha p^ x H)/((1+alpha^2) hbar).  Closed-form Cayley solve with
 * h = a/2: y = m + 2/(1+|h|^2) (u + u x h), u = m x h. */
static void sib_stage(const double* m, const double* p, const double* B, const double* b,
                      double hc, double alpha, double* y_out, int midpoint, int64_t n) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) {
        const double* mi = m + 3 * i; const double* pi = p + 3 * i;
        double Ht[3];
        for (int k = 0; k < 3; k++) Ht[k] = B[3 * i + k] + (b ? b[3 * i + k] : 0.0);
        double np = nrm3(pi);
        double pn[3] = {pi[0], pi[1], pi[2]};
        if (np > 1e-8) { double inv = 1.0 / np; for (int k = 0; k < 3; k++) pn[k] = pi[k] * inv; }
        double pxh[3];
        cross3(pn, Ht, pxh);
        double h[3];
        for (int k = 0; k < 3; k++) h[k] = hc * (Ht[k] + alpha * pxh[k]);
        double u[3], w[3];
        cross3(mi, h, u);
        cross3(u, h, w);
        double h2 = h[0] * h[0] + h[1] * h[1] + h[2] * h[2];
        double c = 2.0 / (1.0 + h2);
        for (int k = 0; k < 3; k++) {
            double y = mi[k] + c * (u[k] + w[k]);
            y_out[3 * i + k] = midpoint ? 0.5 * (mi[k] + y) : y;
        }
    }
}

static void draw_noise(const orc_model* M, const orc_dyn* d, uint32_t step, double sigma, double* b) {
    int64_t N = M->nsite;
    if (d->noise == ORC_NOISE_PHILOX) {
        noise_tables();
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < N; i++) {
            double z[3];
            philox_site(d->seed, step, d->stream, (uint32_t)i, z);
            for (int k = 0; k < 3; k++) b[3 * i + k] = sigma * z[k];
        }
    } else {
        const double* buf = d->inject + (size_t)(step % (uint32_t)d->inject_nbuf) * 3 * N;
        for (int64_t i = 0; i < N; i++)
            for (int k = 0; k < 3; k++) b[3 * i + k] = sigma * buf[(size_t)k * N + i];
    }
}

int orc_run(const orc_model* M, const orc_dyn* d, double* m, int nsteps, double* E_step) {
    int64_t N = M->nsite, n3 = M->n3;
    double* B = (double*)malloc(sizeof(double) * n3);
    double* D1 = (double*)malloc(sizeof(double) * n3);
    double* D2 = (double*)malloc(sizeof(double) * n3);
    double* DT = (double*)calloc((size_t)n3, sizeof(double));
    double* b = (double*)calloc((size_t)n3, sizeof(double));
    double* mt = (double*)malloc(sizeof(double) * n3);
    double* Dint = (double*)malloc(sizeof(double) * n3);
    if (!B || !D1 || !D2 || !DT || !b || !mt || !Dint) return -1;
    double kT = d->temperature * ORC_KB;
    int nloop = d->integrator == ORC_HEUN_MATJES ? 2 : 1;
    double dt = d->timestep / (double)nloop; /* spindynamics.f90:266 */
    int thermal = (kT * d->alpha > 1e-10) && d->noise != ORC_NOISE_OFF && kT > 1e-8;
    double sigma = sqrt(d->alpha * kT * ORC_HBAR / dt);
    for (int s = 0; s < nsteps; s++) {
        uint32_t step = d->step0 + (uint32_t)s;
        if (thermal) draw_noise(M, d, step, sigma, b);
        if (d->integrator == ORC_EULER || d->integrator == ORC_HEUN_MATJES) {
            if (thermal) orc_llg_torque(b, d->alpha, m, DT, N); /* langevin_bath at m_n */
            if (E_step && d->energy_before) field_impl(M, m, B, NULL, NULL, NULL, NULL, &E_step[s]);
            else orc_field(M, m, B, NULL);
            orc_llg_torque(B, d->alpha, m, D1, N);
            if (d->integrator == ORC_EULER) {
                euler_update(m, D1, thermal ? DT : NULL, dt, mt, N);
                memcpy(m, mt, sizeof(double) * n3);
            } else {
                /* stage 1 (Butcher column 2 = [1,1,0]): predictor, no noise */
                euler_update(m, D1, NULL, dt, mt, N);
                /* stage 2 restarts from the predictor (F2) */
                orc_field(M, mt, B, NULL);
                orc_llg_torque(B, d->alpha, mt, D2, N);
                for (int64_t r = 0; r < n3; r++) Dint[r] = 0.5 * D1[r] + 0.5 * D2[r];
                euler_update(mt, Dint, thermal ? DT : NULL, dt, m, N);
            }
        } else {
            double hc = -0.5 * (d->timestep / ORC_HBAR) / (1.0 + d->alpha * d->alpha);
            if (E_step && d->energy_before) field_impl(M, m, B, NULL, NULL, NULL, NULL, &E_step[s]);
            else orc_field(M, m, B, NULL);
            sib_stage(m, m, B, thermal ? b : NULL, hc, d->alpha, mt, 1, N);  /* mt = midpoint */
            orc_field(M, mt, B, NULL);
            sib_stage(m, mt, B, thermal ? b : NULL, hc, d->alpha, D2, 0, N);
            memcpy(m, D2, sizeof(double) * n3);
        }
        if (E_step && !d->energy_before) E_step[s] = orc_energy(M, m);
    }
    free(B); free(D1); free(D2); free(DT); free(b); free(mt); free(Dint);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Minimisation drivers (solvers/minimize.F90)                          */

/* field of one site from the current spins (the single-site counterpart of
 * field_impl; no dipolar term): B_s = -(H + H^T) m |_s - zee b */
static void site_field(const orc_model* M, const double* m, int64_t s, double* B) {
    int nm = M->nmag;
    int64_t cell = s / nm;
    int a = (int)(s % nm);
    for (int k = 0; k < 3; k++) {
        int64_t r = 3 * s + k;
        double hm = 0.0, htm = 0.0;
        for (int64_t j = M->rowptr[r]; j < M->rowptr[r + 1]; j++) hm += M->val[j] * m[M->col[j]];
        for (int64_t j = M->trowptr[r]; j < M->trowptr[r + 1]; j++) htm += M->tval[j] * m[M->tcol[j]];
        double bz = M->in.zeeman_on ? M->zee[a] * M->bfield[3 * cell + k] : 0.0;
        B[k] = -(bz + (htm + hm));
    }
}

/* minimize_run (solvers/minimize.F90:57-166): velocity projection.  The first
 * predictor (euler_minimization with dt^2 and 2 mass, solvers/solver.f90:129-138)
 * is not normalised; later steps keep each spin's norm (euler_o2_minimization,
 * :140-160; a spin whose predictor is shorter than 1e-8 becomes 0).  Returns the
 * iterations run and the last maximum torque |F_i|. */
int orc_minimize_vpo(const orc_model* M, double* m, double dt, double mass, double conv_torque, int64_t niter,
                     int64_t* iters, double* max_torque) {
    int64_t n3 = M->n3, N = M->nsite;
    double* B = (double*)malloc(sizeof(double) * n3);
    double* force = (double*)calloc((size_t)n3, sizeof(double));
    double* vel = (double*)calloc((size_t)n3, sizeof(double));
    if (!B || !force || !vel) { free(B); free(force); free(vel); return -1; }
    orc_field(M, m, B, NULL);
    for (int64_t i = 0; i < N; i++) {
        const double* mi = m + 3 * i;
        double d = mi[0] * B[3 * i] + mi[1] * B[3 * i + 1] + mi[2] * B[3 * i + 2];
        for (int k = 0; k < 3; k++) force[3 * i + k] = -(mi[k] * d - B[3 * i + k]);   /* damping_2V */
    }
    for (int64_t r = 0; r < n3; r++) m[r] = force[r] * (dt * dt) / (mass * 2.0) + m[r];
    int64_t it = 0;
    double maxt = 0.0;
    for (it = 1; it <= niter; it++) {
        orc_field(M, m, B, NULL);
        double dumy = 0.0, fnorm = 0.0;
        for (int64_t i = 0; i < N; i++) {
            const double* mi = m + 3 * i;
            double d = mi[0] * B[3 * i] + mi[1] * B[3 * i + 1] + mi[2] * B[3 * i + 2];
            double F[3], V[3];
            for (int k = 0; k < 3; k++) F[k] = -(mi[k] * d - B[3 * i + k]);
            for (int k = 0; k < 3; k++) V[k] = (force[3 * i + k] + F[k]) / 2.0 * dt / mass + vel[3 * i + k];
            for (int k = 0; k < 3; k++) { force[3 * i + k] = F[k]; vel[3 * i + k] = V[k]; }
            dumy += V[0] * F[0] + V[1] * F[1] + V[2] * F[2];
            fnorm += F[0] * F[0] + F[1] * F[1] + F[2] * F[2];
        }
        for (int64_t r = 0; r < n3; r++) vel[r] = fabs(dumy) > 1e-8 ? dumy * force[r] / fnorm : 0.0;
        maxt = 0.0;
        for (int64_t i = 0; i < N; i++) {
            double s[3];
            for (int k = 0; k < 3; k++)
                s[k] = force[3 * i + k] * (dt * dt) / mass / 2.0 + vel[3 * i + k] * dt + m[3 * i + k];
            double ni = nrm3(m + 3 * i), nf = nrm3(s);
            for (int k = 0; k < 3; k++) m[3 * i + k] = nf > 1e-8 ? s[k] / nf * ni : 0.0;
            double t = nrm3(force + 3 * i);
            if (t > maxt) maxt = t;
        }
        if (conv_torque > maxt) break;
    }
    if (iters) *iters = it > niter ? niter : it;
    if (max_torque) *max_torque = maxt;
    free(B); free(force); free(vel);
    return 0;
}

/* minimize_infdamp_run (solvers/minimize.F90:169-258): every spin is turned onto
 * its normalised local field, the field recomputed from the current neighbours.
 * colors[3] = {1,1,1}: the reference's site order; otherwise the sites of colour
 * (x mod cx) + cx ((y mod cy) + cy (z mod cz)) are visited colour by colour in
 * site order (the order the GPU sweeps).  Returns -2 on a field shorter than 1e-8. */
int orc_minimize_infdamp(const orc_model* M, double* m, double conv_torque, int64_t niter, const int colors[3],
                         int64_t* iters, double* max_torque) {
    const int cx = colors[0], cy = colors[1], cz = colors[2];
    const int ncol = cx * cy * cz;
    const int* L = M->in.lat.L;
    int nm = M->nmag;
    int64_t it = 0;
    double maxt = 0.0;
    for (it = 1; it <= niter; it++) {
        maxt = 0.0;
        for (int col = 0; col < ncol; col++)
            for (int64_t s = 0; s < M->nsite; s++) {
                int64_t cell = s / nm;
                int x = (int)(cell % L[0]), y = (int)((cell / L[0]) % L[1]), z = (int)(cell / ((int64_t)L[0] * L[1]));
                if ((x % cx) + cx * ((y % cy) + cy * (z % cz)) != col) continue;
                double B[3];
                site_field(M, m, s, B);
                double bn = nrm3(B);
                if (bn < 1e-8) return -2;
                for (int k = 0; k < 3; k++) B[k] = B[k] / bn;
                double t[3];
                cross3(m + 3 * s, B, t);
                double tt = fmax(fabs(t[0]), fmax(fabs(t[1]), fabs(t[2])));
                if (tt > maxt) maxt = tt;
                if (nrm3(m + 3 * s) > 1e-8)
                    for (int k = 0; k < 3; k++) m[3 * s + k] = B[k];
            }
        if (maxt < conv_torque) break;
    }
    if (iters) *iters = it > niter ? niter : it;
    if (max_torque) *max_torque = maxt;
    return 0;
}

/* ------------------------------------------------------------------ */
/* Metropolis Monte Carlo (Metropolis-MC/MCstep.f90)                    */

static double mc_u32(uint32_t w) { return ((double)w + 0.5) * (1.0 / 4294967296.0); }

/* sphereft (paratemp-MC/sampling.f90:9-62): cos(theta) uniform in [cos(cone), 1],
 * phi = 2 pi (w2 + 1/2) 2^-32, the new direction rotated from the z frame onto
 * the old spin; sin and cos of phi from the tables of the thermal draw
 * (sincos2pi_word) */
static void mc_sphereft(const double* s, double cos_cone, double u1, uint32_t w2, double* out) {
    double ct = u1 + cos_cone * (1.0 - u1);
    double st = sqrt(1.0 - ct * ct);
    double sph, cph;
    noise_tables();
    sincos2pi_word(w2, &sph, &cph);
    double cti = s[2], rxy2 = s[0] * s[0] + s[1] * s[1], sti = sqrt(rxy2);
    double cpi = 1.0, spi = 0.0;
    if (!(rxy2 < 0.00001)) { cpi = s[0] / sqrt(rxy2); spi = s[1] / sqrt(rxy2); }
    double t = st * sph * cti + ct * sti;
    double n[3] = {-st * cph * spi + t * cpi, st * cph * cpi + t * spi, -st * sph * sti + ct * cti};
    double nn = nrm3(n);
    for (int k = 0; k < 3; k++) out[k] = n[k] / nn;
}

/* the proposals of Metropolis-MC/track_value.f90 (sample_sphere, sample_ising,
 * sample_underrelax, sample_overrelax -> relaxationtype.f90); B = -dE/dm of the site */
static void mc_propose(int proposal, const double* s, const double* B, double cos_cone, double u1, uint32_t w2,
                       double* out) {
    if (proposal == 1) { for (int k = 0; k < 3; k++) out[k] = -s[k]; return; }
    if (proposal == 0) { mc_sphereft(s, cos_cone, u1, w2, out); return; }
    double sb = s[0] * B[0] + s[1] * B[1] + s[2] * B[2], n[3];
    if (proposal == 2) for (int k = 0; k < 3; k++) n[k] = s[k] * (1.0 - sb) + B[k];
    else for (int k = 0; k < 3; k++) n[k] = B[k] - s[k] * (1.0 + sb);
    double nn = nrm3(n);
    for (int k = 0; k < 3; k++) out[k] = n[k] / nn;
}

/* energy change of moving site s to sn: the difference of energy_single
 * (hamiltonian_collection.f90:402-431, pair terms doubled by mult_M_single),
 * written as -d.B_s + d^T H_ss d with d = sn - s; B (out) = -dE/dm of the site */
static double mc_delta_energy(const orc_model* M, const double* m, int64_t s, const double* sn, double* B) {
    site_field(M, m, s, B);
    double d[3] = {sn[0] - m[3 * s], sn[1] - m[3 * s + 1], sn[2] - m[3 * s + 2]};
    double dE = -(d[0] * B[0] + d[1] * B[1] + d[2] * B[2]);
    for (int k = 0; k < 3; k++) {
        int64_t r = 3 * s + k;
        for (int64_t j = M->rowptr[r]; j < M->rowptr[r + 1]; j++) {
            int64_t c = M->col[j];
            if (c >= 3 * s && c < 3 * s + 3) dE += d[k] * M->val[j] * d[c - 3 * s];
        }
    }
    return dE;
}

/* accept (MCstep.f90:75-89) */
static int mc_accept(double kT, double dE, double u) {
    if (dE < 0.0) return 1;
    if (!(kT > 0.0)) return 0;
    return u < exp(fmax(-dE / kT, -200.0));
}

/* cone_update (track_value.f90:149-160) */
static double mc_cone_update(double cone, double rate, double step) {
    if (rate > 0.5 && cone < ORC_PI) return fmin(ORC_PI, cone + step);
    if (rate < 0.5 && cone > 0.01) return fmax(0.01, cone - step);
    return cone;
}

static void mc_keys(uint64_t seed, uint32_t key[2]) { key[0] = (uint32_t)seed; key[1] = (uint32_t)(seed >> 32); }

static void mc_record(const orc_model* M, const double* m, int k, double* E_out, double* M_out) {
    if (E_out) E_out[k] = orc_energy(M, m);
    if (M_out) {
        double a[3] = {0.0, 0.0, 0.0};
        for (int64_t i = 0; i < M->nsite; i++) for (int c = 0; c < 3; c++) a[c] += m[3 * i + c];
        for (int c = 0; c < 3; c++) M_out[3 * k + c] = a[c];
    }
}

int orc_mc_sweeps(const orc_model* M, double* m, orc_mc* p, int nsweeps, const int* site_colour, int ncolours,
                  double* E_out, double* M_out, int64_t* accepted) {
    if (M->nmag != 1 || M->in.dip_on) return -3;
    uint32_t key[2];
    mc_keys(p->seed, key);
    double kT = p->temperature * ORC_KB;
    int64_t acc = 0, N = M->nsite;
    for (int k = 0; k < nsweeps; k++) {
        uint32_t sweep = p->sweep0 + (uint32_t)k;
        double cos_cone = cos(p->cone);
        int64_t acc_sweep = 0;
        for (int col = 0; col < ncolours; col++)
            for (int64_t i = 0; i < N; i++) {
                if (site_colour[i] != col) continue;
                uint32_t c[4] = {(uint32_t)i, sweep, p->stream_id, 0x4D43u}, w[4];
                orc_philox4x32(c, key, w);
                double B[3], sn[3];
                site_field(M, m, i, B);
                mc_propose(p->proposal, m + 3 * i, B, cos_cone, mc_u32(w[0]), w[1], sn);
                double dE = mc_delta_energy(M, m, i, sn, B);
                if (mc_accept(kT, dE, mc_u32(w[2]))) {
                    for (int q = 0; q < 3; q++) m[3 * i + q] = sn[q];
                    acc_sweep++;
                }
            }
        acc += acc_sweep;
        p->accepted_total += acc_sweep;
        p->proposed_total += N;
        if (p->adapt_cone && p->proposal == 0)
            p->cone = mc_cone_update(p->cone, (double)p->accepted_total / (double)p->proposed_total, 1e-4 * (double)N);
        mc_record(M, m, k, E_out, M_out);
    }
    p->sweep0 += (uint32_t)nsweeps;
    if (accepted) *accepted = acc;
    return 0;
}

int orc_mc_random(const orc_model* M, double* m, orc_mc* p, int nsweeps, double* E_out, double* M_out,
                  int64_t* accepted) {
    if (M->in.dip_on) return -3;
    uint32_t key[2];
    mc_keys(p->seed, key);
    double kT = p->temperature * ORC_KB;
    int64_t N = M->nsite, acc = 0;
    /* the tracked totals of track_val (init: H%energy and the summed spins),
     * updated by each accepted move as MCstep.f90:60-68 does */
    double E = orc_energy(M, m), Mg[3] = {0.0, 0.0, 0.0};
    for (int64_t i = 0; i < N; i++) for (int c = 0; c < 3; c++) Mg[c] += m[3 * i + c];
    for (int k = 0; k < nsweeps; k++) {
        uint32_t sweep = p->sweep0 + (uint32_t)k;
        for (int64_t t = 0; t < N; t++) {
            uint32_t c[4] = {(uint32_t)t, sweep, p->stream_id, 0x52534D43u}, w[4];
            orc_philox4x32(c, key, w);
            /* choose_spin (choosespin.f90:19-21): iomp = 1 + INT(Choice*(N-1)) */
            int64_t i = (int64_t)(mc_u32(w[0]) * (double)(N - 1));
            if (p->proposal == 0 && p->adapt_cone)
                p->cone = mc_cone_update(p->cone,
                                         p->proposed_total ? (double)p->accepted_total / (double)p->proposed_total : 0.0,
                                         1e-4);
            double B[3], sn[3];
            site_field(M, m, i, B);
            mc_propose(p->proposal, m + 3 * i, B, cos(p->cone), mc_u32(w[1]), w[2], sn);
            double dE = mc_delta_energy(M, m, i, sn, B);
            p->proposed_total++;
            if (mc_accept(kT, dE, mc_u32(w[3]))) {
                for (int q = 0; q < 3; q++) { Mg[q] += sn[q] - m[3 * i + q]; m[3 * i + q] = sn[q]; }
                E += dE;
                acc++;
                p->accepted_total++;
            }
        }
        if (E_out) E_out[k] = E;
        if (M_out) for (int q = 0; q < 3; q++) M_out[3 * k + q] = Mg[q];
    }
    p->sweep0 += (uint32_t)nsweeps;
    if (accepted) *accepted = acc;
    return 0;
}

void orc_set_threads(int n) { omp_set_num_threads(n > 0 ? n : omp_get_num_procs()); }

/* ------------------------------------------------------------------ */
/* GNEB minimum-energy path (GNEB/gneb_utils.f90:19-240 find_path)      */

static double gn_ang(const double* a, const double* b) {
    double c[3];
    cross3(a, b, c);
    return atan2(nrm3(c), a[0] * b[0] + a[1] * b[1] + a[2] * b[2]);
}

/* the_path (GNEB/path.f90:10-29): cumulative geodesic length of the images */
static void gn_path(const double* img, int nim, int64_t N, double* pl) {
    pl[0] = 0.0;
    for (int i = 1; i < nim; i++) {
        double t = 0.0;
        for (int64_t s = 0; s < N; s++) {
            double l = gn_ang(img + ((int64_t)(i - 1) * N + s) * 3, img + ((int64_t)i * N + s) * 3);
            t += l * l;
        }
        pl[i] = pl[i - 1] + sqrt(t);
    }
}

/* tau minus its component along each spin, normalised over the image */
static void gn_project_normalise(const double* m, double* tau, int64_t N) {
    double t2 = 0.0;
    for (int64_t s = 0; s < N; s++) {
        double* t = tau + 3 * s;
        const double* ms = m + 3 * s;
        double d = t[0] * ms[0] + t[1] * ms[1] + t[2] * ms[2];
        for (int k = 0; k < 3; k++) { t[k] -= d * ms[k]; t2 += t[k] * t[k]; }
    }
    double inv = 1.0 / sqrt(t2);
    for (int64_t r = 0; r < 3 * N; r++) tau[r] *= inv;
}

/* lattice_single (tangent.f90:169-180) and lattice_special (:89-124) */
static void gn_tang_single(const double* img, int nim, int64_t N, int im, double* tau) {
    int u1 = im + 1 < nim ? im + 1 : im, u2 = im > 0 ? im - 1 : im;
    for (int64_t r = 0; r < 3 * N; r++) tau[r] = img[(int64_t)u1 * 3 * N + r] - img[(int64_t)u2 * 3 * N + r];
    gn_project_normalise(img + (int64_t)im * 3 * N, tau, N);
}
static void gn_tang_special(const double* img, int64_t N, int im, const double* u, double* tau) {
    double u1 = u[im - 1], u2 = u[im], u3 = u[im + 1];
    const double *a = img + (int64_t)(im - 1) * 3 * N, *b = img + (int64_t)im * 3 * N, *c = img + (int64_t)(im + 1) * 3 * N;
    if (u3 > u2 && u2 > u1) {
        for (int64_t r = 0; r < 3 * N; r++) tau[r] = c[r] - b[r];
    } else if (u1 > u2 && u2 > u3) {
        for (int64_t r = 0; r < 3 * N; r++) tau[r] = b[r] - a[r];
    } else {
        double dmax = fabs(u3 - u2), dmin = fabs(u1 - u2);
        if (dmax < dmin) { double t = dmax; dmax = dmin; dmin = t; }
        double wp = u3 > u1 ? dmax : dmin, wm = u3 > u1 ? dmin : dmax;
        for (int64_t r = 0; r < 3 * N; r++) tau[r] = wp * (c[r] - b[r]) + wm * (b[r] - a[r]);
    }
    gn_project_normalise(b, tau, N);
}

/* rotate_vector_arr (utilities/rotation.f90): v cos + sin (v x ax) + (1 - cos)(ax.v) ax */
static void gn_rotate(const double* v, const double* ax, double ang, double* out) {
    double t = ax[0] * v[0] + ax[1] * v[1] + ax[2] * v[2], s = sin(ang), c = cos(ang);
    out[0] = v[0] * c + s * (ax[2] * v[1] - ax[1] * v[2]) + (1.0 - c) * t * ax[0];
    out[1] = v[1] * c + s * (ax[0] * v[2] - ax[2] * v[0]) + (1.0 - c) * t * ax[1];
    out[2] = v[2] * c + s * (ax[1] * v[0] - ax[0] * v[1]) + (1.0 - c) * t * ax[2];
}

/* the field projected on each spin's tangent plane, and the energy, of every image */
static void gn_fields(const orc_model* M, const double* img, int i0, int i1, int64_t N, double* F, double* E) {
    for (int i = i0; i < i1; i++) {
        const double* m = img + (int64_t)i * 3 * N;
        double* f = F + (int64_t)i * 3 * N;
        orc_field(M, m, f, NULL);
        E[i] = orc_energy(M, m);
        for (int64_t s = 0; s < N; s++) {
            double d = f[3 * s] * m[3 * s] + f[3 * s + 1] * m[3 * s + 1] + f[3 * s + 2] * m[3 * s + 2];
            for (int k = 0; k < 3; k++) f[3 * s + k] -= d * m[3 * s + k];
        }
    }
}

/* GNEB forces of the interior images: the perpendicular part of the force plus the
 * spring force along the energy-weighted tangent; at the climbing image ci (-1:
 * none) the force with its component along the tangent reversed and no spring
 * (gneb_utils.f90:105-111); fpp the force along the simple tangent (the energy
 * derivative along the path) */
static void gn_gneb_forces(const double* img, int nim, int64_t N, const double* E, const double* pl, double spring,
                           int ci, double* F, double* fpp, double* tau, double* tau_i) {
    for (int im = 1; im < nim - 1; im++) {
        double* f = F + (int64_t)im * 3 * N;
        gn_tang_special(img, N, im, E, tau);
        gn_tang_single(img, nim, N, im, tau_i);
        double fp = 0.0, fi = 0.0;
        for (int64_t r = 0; r < 3 * N; r++) { fi += f[r] * tau_i[r]; fp += f[r] * tau[r]; }
        fpp[im] = fi;
        if (im == ci) {
            for (int64_t r = 0; r < 3 * N; r++) f[r] = f[r] - 2.0 * tau[r] * fp;
            continue;
        }
        double sp = spring * (pl[im + 1] + pl[im - 1] - 2.0 * pl[im]);
        for (int64_t r = 0; r < 3 * N; r++) f[r] = f[r] - tau[r] * fp + sp * tau[r];
    }
}

/* maxloc: the first image of highest energy */
static int gn_maxloc(const double* E, int nim) {
    int c = 0;
    for (int i = 1; i < nim; i++)
        if (E[i] > E[c]) c = i;
    return c;
}

int orc_gneb_find_path(const orc_model* M, double* img, int nim, double spring, double dt, double mass, double ftol,
                       int64_t itrmax, int en_zero, int climb, double* rx, double* ene, double* dene, int64_t* iters,
                       double* fchk_out, int* ci_out) {
    if (M->nmag != 1 || nim < 3) return -3;
    const int64_t N = M->nsite, n3 = 3 * N, tot = (int64_t)nim * n3;
    double *F1 = calloc((size_t)tot, sizeof(double)), *F2 = calloc((size_t)tot, sizeof(double));
    double *vel = calloc((size_t)tot, sizeof(double)), *ax = calloc((size_t)tot, sizeof(double));
    double *ang = calloc((size_t)nim * N, sizeof(double)), *tau = malloc(sizeof(double) * n3);
    double *tau_i = malloc(sizeof(double) * n3), *E = calloc((size_t)nim, sizeof(double));
    double *fpp = calloc((size_t)nim, sizeof(double)), *pl = calloc((size_t)nim, sizeof(double));
    if (!F1 || !F2 || !vel || !ax || !ang || !tau || !tau_i || !E || !fpp || !pl) return -1;
    gn_path(img, nim, N, pl);
    gn_fields(M, img, 0, nim, N, F1, E);
    double eref = en_zero == 'I' ? E[0] : (en_zero == 'F' ? E[nim - 1] : 0.0);
    int ci = climb ? gn_maxloc(E, nim) : -1;
    gn_gneb_forces(img, nim, N, E, pl, spring, ci, F1, fpp, tau, tau_i);
    double fchk = 0.0;
    for (int64_t r = 0; r < tot; r++) fchk = fmax(fchk, fabs(F1[r]));
    int64_t itr = 0, done = 0;
    for (itr = 1; itr <= itrmax; itr++) {
        /* move the interior images: r = m + v dt + F/(2 mass) dt^2, normalised;
         * the rotation axis m x F1 and the angle of each spin's move kept */
        for (int im = 1; im < nim - 1; im++)
            for (int64_t s = 0; s < N; s++) {
                int64_t o = ((int64_t)im * N + s) * 3;
                double* m = img + o;
                double fn[3] = {F1[o], F1[o + 1], F1[o + 2]}, a[3], r[3];
                double nf = nrm3(fn);
                if (nf > 1e-30) for (int k = 0; k < 3; k++) fn[k] /= nf;
                cross3(m, fn, a);
                double na = nrm3(a);
                if (na > DBL_EPSILON) for (int k = 0; k < 3; k++) a[k] /= na;
                for (int k = 0; k < 3; k++) { ax[o + k] = a[k]; r[k] = m[k] + vel[o + k] * dt + 0.5 * F1[o + k] / mass * dt * dt; }
                double nr = nrm3(r);
                if (nr > 1e-30) for (int k = 0; k < 3; k++) r[k] /= nr;
                ang[(int64_t)im * N + s] = gn_ang(r, m);
                for (int k = 0; k < 3; k++) m[k] = r[k];
            }
        gn_fields(M, img, 1, nim - 1, N, F2, E);
        gn_path(img, nim, N, pl);
        if (climb) ci = gn_maxloc(E, nim);
        gn_gneb_forces(img, nim, N, E, pl, spring, ci, F2, fpp, tau, tau_i);
        /* parallel transport of the velocity and the old force, velocity Verlet */
        for (int im = 1; im < nim - 1; im++)
            for (int64_t s = 0; s < N; s++) {
                int64_t o = ((int64_t)im * N + s) * 3;
                double vr[3], fr[3], a = ang[(int64_t)im * N + s];
                gn_rotate(vel + o, ax + o, a, vr);
                gn_rotate(F1 + o, ax + o, a, fr);
                for (int k = 0; k < 3; k++) vel[o + k] = vr[k] + 0.5 * (fr[k] + F2[o + k]) / mass * dt;
            }
        /* velocity projection on the force (VPO) */
        double fv = 0.0, fd = 0.0;
        for (int64_t r = 0; r < tot; r++) { fv += vel[r] * F2[r]; fd += F2[r] * F2[r]; }
        fv /= nim;
        fd /= nim;
        for (int64_t r = 0; r < tot; r++) vel[r] = fv < 0.0 ? 0.0 : F2[r] * fv / fd;
        fchk = 0.0;
        for (int64_t r = 0; r < tot; r++) { F1[r] = F2[r]; fchk = fmax(fchk, fabs(F2[r])); }
        done = itr;
        if (fchk < ftol) break;
    }
    /* the energy derivative along the path at the end images, from their forces */
    gn_tang_single(img, nim, N, 0, tau_i);
    fpp[0] = 0.0;
    for (int64_t r = 0; r < n3; r++) fpp[0] += F1[r] * tau_i[r];
    gn_tang_single(img, nim, N, nim - 1, tau_i);
    fpp[nim - 1] = 0.0;
    for (int64_t r = 0; r < n3; r++) fpp[nim - 1] += F1[(int64_t)(nim - 1) * n3 + r] * tau_i[r];
    for (int i = 0; i < nim; i++) { rx[i] = pl[i]; ene[i] = E[i] - eref; dene[i] = -fpp[i]; }
    if (iters) *iters = done;
    if (fchk_out) *fchk_out = fchk;
    if (ci_out) *ci_out = ci;
    free(F1); free(F2); free(vel); free(ax); free(ang); free(tau); free(tau_i); free(E); free(fpp); free(pl);
    return 0;
}
