/*
 * oracle/bsr_oracle.c -- CPU restatement of the BSR radial + assembly hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: it is loaded by tests/,
 * by __graft_entry__.smoke() and by bench.py's cpu_baseline / reference leg,
 * and by nothing else.  The shipped library (bsr_b200/libbsrgpu.so) never
 * links, loads or calls it.
 *
 * It restates, single-threaded and in the reference's own loop order, the
 * Fortran routines of jagot/bsr that the GPU path replaces (paths relative to
 * the reference's src/ tree):
 *
 *   gauss            libs/BS/gauss.f90:2            (nodes computed, see below)
 *   mkgrid/mkgrid1   libs/BS/define_grid.f90:86,213
 *   vbsplvd/vbsplvb  libs/BS/vbsplvd.f90:3,170      (de Boor's bsplvd/bsplvb)
 *   initvb/initas    libs/BS/define_spline.f90:67,133  mdb1 :184  mdb2 :214
 *   mrm              libs/BS/mrm.f90:2
 *   zfacsb/bhwf      libs/BS/bhwf.f90:2,73  vhwf :119  hnorm1 :202
 *   vinty            libs/BS/vinty.f90:2
 *   moments/moment   libs/BS/moments.f90:2,76
 *   rk_moments       libs/BS/rk_moments.f90:2  rk_pdiag :56  rk_triang :105
 *   mrk_cell         libs/BS/mrk_cell.f90:2
 *   density          libs/BS/density.f90:2
 *   convol           libs/BS/convol.f90:2  (all 12 icase/sym cases)
 *   SUM_AmB          libs/BS/sum_amb.f90:2
 *   bav              libs/BS/bav.f90:2
 *   bvmv             libs/BS/bvmv.f90:2
 *   rk               libs/BS/rk.f90:2
 *   rkd/rke/rkv      libs/BS/TEST_BS/test_bs.f90:2177,2216,1091 (with INT_de
 *                    libs/BS/int_de.f90:2 and INT_v libs/BS/int_v.f90:2)
 *   INT_core (no closed shells)  bsr/BSR_MAT3/l_core.f90:174
 *   I_data Case(6..9), UPDATE_HX/HL/CF, SUB1 symmetrisation
 *                    bsr/BSR_MAT3/I_data.f90:192, mod_intmat.f90:69,131,245,
 *                    sub1.f90:72-84,178-191
 *
 * Storage follows the Fortran arrays exactly (column-major, 0-based here):
 *   t[0..ns+ks-1];  gr/grm/grw (nv,ks): [iv + nv*m];
 *   bsp/bsq (nv+1,ks,ks): [iv + (nv+1)*(m + ks*ith)];  bspd adds a last index d=0,1;
 *   band matrices (ns,ks) lower-column storage: element (i, i+jcol-ks+1) at [i + ns*jcol];
 *   rkb (ns,ns,ldp,ldp): [i + ns*(j + ns*(ip + ldp*jp))].
 *
 * The Gauss-Legendre nodes are computed by Newton iteration on P_k instead of
 * being read from the reference's 15-digit table; the two agree to ~1e-16.
 *
 * Compile with -ffp-contract=off: the reference (gfortran -O2, x86-64) does
 * not fuse multiply-adds, and neither does this restatement.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>

#define MAXKS 16

/* ------------------------------------------------------------------------ */
/* Gauss-Legendre nodes and weights on [0,1], ascending nodes               */
/* ------------------------------------------------------------------------ */
int orc_gauss(int k, double *x, double *w)
{
    if (k < 1 || k > 64) return -1;
    for (int i = 0; i < k; i++) {
        double z = cos(M_PI * (i + 0.75) / (k + 0.5));
        double p = 0.0, pm = 0.0, dp = 1.0;
        for (int it = 0; it < 200; it++) {
            double p0 = 1.0, p1 = z;
            for (int j = 2; j <= k; j++) {
                double p2 = ((2.0 * j - 1.0) * z * p1 - (j - 1.0) * p0) / j;
                p0 = p1; p1 = p2;
            }
            p = p1; pm = p0;
            dp = k * (z * p - pm) / (z * z - 1.0);
            double dz = p / dp;
            z -= dz;
            if (fabs(dz) <= 1e-17) break;
        }
        {   /* derivative at the converged node for the weight */
            double p0 = 1.0, p1 = z;
            for (int j = 2; j <= k; j++) {
                double p2 = ((2.0 * j - 1.0) * z * p1 - (j - 1.0) * p0) / j;
                p0 = p1; p1 = p2;
            }
            if (k == 1) { p1 = z; p0 = 1.0; }
            dp = k * (z * p1 - p0) / (z * z - 1.0);
        }
        x[i] = 0.5 * (1.0 - z);
        w[i] = 1.0 / ((1.0 - z * z) * dp * dp);
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* knot grids                                                               */
/* ------------------------------------------------------------------------ */
/* grid_type 0 (define_grid.f90:86 mkgrid).  t must hold cap doubles. */
int orc_mkgrid0(int ks, double z, double h, double hmax, double rmax,
                double *t, int cap, int *ns_out, int *ml_out, int *me_out, double *h_out)
{
    double h0 = h;
    int ml = (int)(1.0 / h + 0.1);
    h = 1.0 / ml;
    double hp1 = 1.0 + h;
    double tmax = z * rmax;
    double hmx = z * hmax;
    double a = log(hmx / h) / log(hp1) + 1.0;
    int me1 = (int)(a > 0.0 ? a : 0.0);
    int me2 = (int)(log(tmax) / log(hp1) + 1.0);
    int me, m;
    double h2 = 0.0;
    if (me2 <= me1) { me = me2; m = 0; }
    else {
        me = me1;
        double tx = 1.0;
        for (int i = 0; i < me; i++) tx *= hp1;
        h2 = h * tx / hp1;
        m = (int)lround((tmax - tx) / h2);
    }
    int n = ml + me + m + ks - 1;
    int ns = n, nt = ns + ks;
    if (nt > cap) return -1;
    for (int i = 0; i < nt; i++) t[i] = 0.0;
    /* Fortran 1-based: t(i) for i = ks+1..ks+ml, etc. */
    for (int i = ks + 1; i <= ks + ml; i++) t[i - 1] = t[i - 2] + h0;
    for (int i = ks + ml + 1; i <= ks + me + ml; i++) t[i - 1] = t[i - 2] * hp1;
    for (int i = ks + me + ml + 1; i <= n + 1; i++) t[i - 1] = t[i - 2] + h2;
    for (int i = n + 2; i <= nt; i++) t[i - 1] = t[n];
    for (int i = 0; i < nt; i++) t[i] = t[i] / z;
    *ns_out = ns; *ml_out = ml; *me_out = me; *h_out = h;
    return 0;
}

/* grid_type 1 (define_grid.f90:213 mkgrid1).  t must hold cap doubles. */
int orc_mkgrid1(int ks, double z, double h, double hmax, double rmax,
                double *t, int cap, int *ns_out, int *ml_out, int *me_out, double *h_out)
{
    rmax = rmax * z;
    hmax = hmax * z;
    int nt = (int)((rmax / h + 1 + ks) * 2);
    if (nt + ks > cap) return -1;
    for (int i = 0; i < cap; i++) t[i] = 0.0;
    int ns = ks;                         /* 1-based count */
#define T1(i) t[(i) - 1]
    int ml = (int)(1.0 / h + 0.5);
    h = 1.0 / ml;
    for (int i = 1; i <= ml; i++) { ns++; T1(ns) = T1(ns - 1) + h; }
    if (hmax < h) hmax = h;
    int me = 0;
    for (;;) {
        T1(ns + 1) = T1(ns) * (1.0 + h);
        if (T1(ns + 1) - T1(ns) > hmax) break;
        ns++;
        if (T1(ns) > rmax) break;
        me++;
    }
    if (T1(ns) < rmax) {
        for (;;) {
            T1(ns + 1) = T1(ns) + hmax;
            ns++;
            if (T1(ns) >= rmax) break;
        }
    }
    if (T1(ns) > rmax) {
        ns--; me--;
        for (int i = ns + 1; i <= ns + ks; i++) T1(i) = rmax;
        T1(ns) = (T1(ns + 1) + T1(ns - 1)) / 2.0;
    }
#undef T1
    for (int i = 0; i < ns + ks; i++) t[i] = t[i] / z;
    *ns_out = ns; *ml_out = ml; *me_out = me; *h_out = h;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* de Boor's B-spline recurrences (vbsplvd.f90:3, :170), one point          */
/* ------------------------------------------------------------------------ */
typedef struct { int j; double deltal[MAXKS + 1], deltar[MAXKS + 1]; } bvb_state;

/* left is the 0-based index of the knot with t[left] <= x <= t[left+1];
   biatx[0..jout-1] receives B_{left-jout+1..left} of order jout. */
static void bsplvb(const double *t, int jhigh, int index, double x, int left,
                   double *biatx, bvb_state *st)
{
    if (index == 1) {
        st->j = 1;
        biatx[0] = 1.0;
        if (st->j >= jhigh) return;
    }
    for (;;) {
        int j = st->j, jp1 = j + 1;
        st->deltar[j - 1] = t[left + j] - x;
        st->deltal[j - 1] = x - t[left + 1 - j];
        double saved = 0.0;
        for (int i = 1; i <= j; i++) {
            double term = biatx[i - 1] / (st->deltar[i - 1] + st->deltal[jp1 - i - 1]);
            biatx[i - 1] = saved + st->deltar[i - 1] * term;
            saved = st->deltal[jp1 - i - 1] * term;
        }
        biatx[jp1 - 1] = saved;
        st->j = jp1;
        if (st->j >= jhigh) break;
    }
}

/* db[(j) + k*(m)] = m-th derivative (m < nderiv) of the j-th (0-based) of the
   k B-splines that are nonzero on [t[left], t[left+1]] at x. */
void orc_bsplvd(const double *t, int k, double x, int left, int nderiv, double *db)
{
    double a[MAXKS * MAXKS];
    bvb_state st;
#define DB(j, m) db[((j) - 1) + k * ((m) - 1)]
#define A(i, j) a[((i) - 1) + k * ((j) - 1)]
    int mhigh = nderiv < k ? nderiv : k;
    if (mhigh < 1) mhigh = 1;
    int kp1 = k + 1;
    bsplvb(t, kp1 - mhigh, 1, x, left, db, &st);
    if (mhigh == 1) return;
    int ideriv = mhigh;
    for (int m = 2; m <= mhigh; m++) {
        int jp1mid = 1;
        for (int j = ideriv; j <= k; j++) { DB(j, ideriv) = DB(jp1mid, 1); jp1mid++; }
        ideriv--;
        bsplvb(t, kp1 - ideriv, 2, x, left, db, &st);
    }
    int jlow = 1;
    for (int i = 1; i <= k; i++) {
        for (int j = jlow; j <= k; j++) A(j, i) = 0.0;
        jlow = i;
        A(i, i) = 1.0;
    }
    for (int m = 2; m <= mhigh; m++) {
        int kp1mm = kp1 - m;
        double fkp1mm = (double)kp1mm;
        int il = left, i = k;
        for (int ld = 1; ld <= kp1mm; ld++) {
            double factor = fkp1mm / (t[il + kp1mm] - t[il]);
            for (int j = 1; j <= i; j++) A(i, j) = (A(i, j) - A(i - 1, j)) * factor;
            il--; i--;
        }
        for (int ii = 1; ii <= k; ii++) {
            double sum = 0.0;
            int jl = ii > m ? ii : m;
            for (int j = jl; j <= k; j++) sum = sum + A(j, ii) * DB(j, m);
            DB(ii, m) = sum;
        }
    }
#undef DB
#undef A
}

/* ------------------------------------------------------------------------ */
/* basis (spline_param + spline_grid + spline_galerkin module state)        */
/* ------------------------------------------------------------------------ */
typedef struct {
    int ks, ns, nv, ml, me;
    double h;
    double *t;
    double gx[MAXKS], gw[MAXKS];
    double *gr, *grm, *grw;
    double *bsp, *bsq, *bspd;
    double *sb, *r1, *rm1, *rm2, *rm3, *db1, *db2;
} orc_basis;

#define GR(b, iv, m)        (b)->gr[(iv) + (size_t)(b)->nv * (m)]
#define GRM(b, iv, m)       (b)->grm[(iv) + (size_t)(b)->nv * (m)]
#define GRW(b, iv, m)       (b)->grw[(iv) + (size_t)(b)->nv * (m)]
#define BSP(b, iv, m, ith)  (b)->bsp[(iv) + (size_t)((b)->nv + 1) * ((m) + (b)->ks * (ith))]
#define BSQ(b, iv, m, ith)  (b)->bsq[(iv) + (size_t)((b)->nv + 1) * ((m) + (b)->ks * (ith))]
#define BSPD(b, iv, m, ith, d) (b)->bspd[(iv) + (size_t)((b)->nv + 1) * ((m) + (b)->ks * ((ith) + (b)->ks * (d)))]
#define BAND(x, ns, i, j)   (x)[(i) + (size_t)(ns) * (j)]

static void initvb(orc_basis *b)
{
    int ks = b->ks, nv = b->nv, ns = b->ns;
    double db[MAXKS * 3];
    for (int m = 0; m < ks; m++) {
        for (int iv = 0; iv < nv; iv++) {
            double tl = b->t[iv + ks - 1], tr = b->t[iv + ks];
            GR(b, iv, m) = (tr - tl) * b->gx[m] + tl;
            GRM(b, iv, m) = 1.0 / GR(b, iv, m);
            GRW(b, iv, m) = (tr - tl) * b->gw[m];
            orc_bsplvd(b->t, ks, GR(b, iv, m), iv + ks - 1, 3, db);
            for (int ith = 0; ith < ks; ith++) {
                BSP(b, iv, m, ith) = db[ith];
                BSPD(b, iv, m, ith, 0) = db[ith + ks];
                BSPD(b, iv, m, ith, 1) = db[ith + 2 * ks];
                BSQ(b, iv, m, ith) = BSPD(b, iv, m, ith, 0) - GRM(b, iv, m) * BSP(b, iv, m, ith);
            }
        }
    }
    orc_bsplvd(b->t, ks, b->t[ns], ns - 1, 3, db);
    for (int ith = 0; ith < ks; ith++) {
        BSP(b, nv, 0, ith) = db[ith];
        BSPD(b, nv, 0, ith, 0) = db[ith + ks];
        BSPD(b, nv, 0, ith, 1) = db[ith + 2 * ks];
        BSQ(b, nv, 0, ith) = BSPD(b, nv, 0, ith, 0) - BSP(b, nv, 0, ith) / b->t[ns];
    }
}

/* mrm.f90:2  <B_i | r^mm | B_j> in lower-band storage */
void orc_mrm(const orc_basis *b, int mm, double *rm)
{
    int ks = b->ks, ns = b->ns, nv = b->nv;
    memset(rm, 0, sizeof(double) * ns * ks);
    for (int ith = 0; ith < ks; ith++)
        for (int jth = 0; jth <= ith; jth++) {
            int jcol = jth - ith + ks - 1;
            for (int iv = 0; iv < nv; iv++) {
                int irow = iv + ith;
                double s = 0.0;
                for (int m = 0; m < ks; m++) {
                    double v;
                    double wb = GRW(b, iv, m) * BSP(b, iv, m, ith);
                    if (mm == 0) v = wb * BSP(b, iv, m, jth);
                    else if (mm == -1) v = wb * GRM(b, iv, m) * BSP(b, iv, m, jth);
                    else if (mm <= -2) {
                        double g = GRM(b, iv, m), p = g;
                        for (int q = 1; q < -mm; q++) p = p * g;
                        v = wb * p * BSP(b, iv, m, jth);
                    } else if (mm == 1) v = wb * GR(b, iv, m) * BSP(b, iv, m, jth);
                    else {
                        double g = GR(b, iv, m), p = g;
                        for (int q = 1; q < mm; q++) p = p * g;
                        v = wb * p * BSP(b, iv, m, jth);
                    }
                    s = s + v;
                }
                BAND(rm, ns, irow, jcol) = BAND(rm, ns, irow, jcol) + s;
            }
        }
}

/* define_spline.f90:184 mdb1, :214 mdb2 */
static void mdb(const orc_basis *b, int d, double *x)
{
    int ks = b->ks, ns = b->ns, nv = b->nv;
    memset(x, 0, sizeof(double) * ns * ks);
    for (int ith = 0; ith < ks; ith++)
        for (int jth = 0; jth <= ith; jth++) {
            int jcol = jth - ith + ks - 1;
            for (int iv = 0; iv < nv; iv++) {
                int irow = iv + ith;
                double s = 0.0;
                for (int m = 0; m < ks; m++)
                    s = s + GRW(b, iv, m) * BSP(b, iv, m, ith) * BSPD(b, iv, m, jth, d);
                BAND(x, ns, irow, jcol) = BAND(x, ns, irow, jcol) + s;
            }
        }
    if (d == 1) {
        double s = 0.0;
        for (int m = 0; m < ks; m++)
            s = s + GRW(b, nv - 1, m) * BSP(b, nv - 1, m, ks - 2) * BSPD(b, nv - 1, m, ks - 1, 1);
        x[0] = x[0] + s;
    }
}

orc_basis *orc_basis_new(int ks, int ns, const double *t, int ml, int me, double h)
{
    if (ks < 2 || ks > MAXKS || ns < ks) return NULL;
    orc_basis *b = (orc_basis *)calloc(1, sizeof(orc_basis));
    b->ks = ks; b->ns = ns; b->nv = ns - ks + 1; b->ml = ml; b->me = me; b->h = h;
    int nv = b->nv;
    b->t = (double *)malloc(sizeof(double) * (ns + ks));
    memcpy(b->t, t, sizeof(double) * (ns + ks));
    orc_gauss(ks, b->gx, b->gw);
    b->gr = (double *)calloc((size_t)nv * ks, sizeof(double));
    b->grm = (double *)calloc((size_t)nv * ks, sizeof(double));
    b->grw = (double *)calloc((size_t)nv * ks, sizeof(double));
    size_t nb = (size_t)(nv + 1) * ks * ks;
    b->bsp = (double *)calloc(nb, sizeof(double));
    b->bsq = (double *)calloc(nb, sizeof(double));
    b->bspd = (double *)calloc(nb * 2, sizeof(double));
    size_t nband = (size_t)ns * ks;
    b->sb = (double *)calloc(nband, sizeof(double));
    b->r1 = (double *)calloc(nband, sizeof(double));
    b->rm1 = (double *)calloc(nband, sizeof(double));
    b->rm2 = (double *)calloc(nband, sizeof(double));
    b->rm3 = (double *)calloc(nband, sizeof(double));
    b->db1 = (double *)calloc(nband, sizeof(double));
    b->db2 = (double *)calloc(nband, sizeof(double));
    initvb(b);
    mdb(b, 0, b->db1);
    mdb(b, 1, b->db2);
    orc_mrm(b, 0, b->sb);
    orc_mrm(b, 1, b->r1);
    orc_mrm(b, -1, b->rm1);
    orc_mrm(b, -2, b->rm2);
    orc_mrm(b, -3, b->rm3);
    return b;
}

void orc_basis_free(orc_basis *b)
{
    if (!b) return;
    free(b->t); free(b->gr); free(b->grm); free(b->grw);
    free(b->bsp); free(b->bsq); free(b->bspd);
    free(b->sb); free(b->r1); free(b->rm1); free(b->rm2); free(b->rm3);
    free(b->db1); free(b->db2);
    free(b);
}

int orc_basis_dims(const orc_basis *b, int *out)
{
    out[0] = b->ks; out[1] = b->ns; out[2] = b->nv; out[3] = b->ml; out[4] = b->me;
    return 0;
}

/* copy a named table out: 0 gr,1 grm,2 grw,3 bsp,4 bsq,5 bspd,6 sb,7 r1,8 rm1,
   9 rm2,10 rm3,11 db1,12 db2,13 gx,14 gw */
int orc_basis_get(const orc_basis *b, int which, double *out)
{
    size_t nvk = (size_t)b->nv * b->ks, nb = (size_t)(b->nv + 1) * b->ks * b->ks,
           nband = (size_t)b->ns * b->ks;
    switch (which) {
    case 0: memcpy(out, b->gr, nvk * 8); break;
    case 1: memcpy(out, b->grm, nvk * 8); break;
    case 2: memcpy(out, b->grw, nvk * 8); break;
    case 3: memcpy(out, b->bsp, nb * 8); break;
    case 4: memcpy(out, b->bsq, nb * 8); break;
    case 5: memcpy(out, b->bspd, nb * 16); break;
    case 6: memcpy(out, b->sb, nband * 8); break;
    case 7: memcpy(out, b->r1, nband * 8); break;
    case 8: memcpy(out, b->rm1, nband * 8); break;
    case 9: memcpy(out, b->rm2, nband * 8); break;
    case 10: memcpy(out, b->rm3, nband * 8); break;
    case 11: memcpy(out, b->db1, nband * 8); break;
    case 12: memcpy(out, b->db2, nband * 8); break;
    case 13: memcpy(out, b->gx, b->ks * 8); break;
    case 14: memcpy(out, b->gw, b->ks * 8); break;
    default: return -1;
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* dense symmetric positive-definite helpers (stand-in for DPBTRF/DPBTRS)   */
/* ------------------------------------------------------------------------ */
static int chol_solve(int n, double *a, double *x)
{
    /* a: n x n column-major full symmetric; lower Cholesky in place */
    for (int j = 0; j < n; j++) {
        double s = a[j + (size_t)n * j];
        for (int k = 0; k < j; k++) s -= a[j + (size_t)n * k] * a[j + (size_t)n * k];
        if (!(s > 0.0)) return -(j + 1);
        double d = sqrt(s);
        a[j + (size_t)n * j] = d;
        for (int i = j + 1; i < n; i++) {
            double v = a[i + (size_t)n * j];
            for (int k = 0; k < j; k++) v -= a[i + (size_t)n * k] * a[j + (size_t)n * k];
            a[i + (size_t)n * j] = v / d;
        }
    }
    for (int i = 0; i < n; i++) {
        double v = x[i];
        for (int k = 0; k < i; k++) v -= a[i + (size_t)n * k] * x[k];
        x[i] = v / a[i + (size_t)n * i];
    }
    for (int i = n - 1; i >= 0; i--) {
        double v = x[i];
        for (int k = i + 1; k < n; k++) v -= a[k + (size_t)n * i] * x[k];
        x[i] = v / a[i + (size_t)n * i];
    }
    return 0;
}

/* bhwf.f90:202 hnorm1 */
static double hnorm1(int n, int l, double z)
{
    int m = l + l + 1;
    double a = n + l, b = m, t = a, d = b;
    m = m - 1;
    for (int i = 1; i <= m; i++) { a = a - 1.0; b = b - 1.0; t = t * a; d = d * b; }
    return sqrt(z * t) / (n * d);
}

/* bhwf.f90:119 vhwf */
static void vhwf(int n, int l, double z, int nr, const double *r, double *vh)
{
    int k = n - l - 1;
    double factor = hnorm1(n, l, z);
    double *w = (double *)malloc(sizeof(double) * nr), *p = (double *)malloc(sizeof(double) * nr);
    for (int i = 0; i < nr; i++) w[i] = -2.0 * z * r[i] / n;
    int nm = nr;
    while (nm >= 1 && w[nm - 1] < -150.0) { vh[nm - 1] = 0.0; nm--; }
    for (int i = 0; i < nm; i++) p[i] = 1.0;
    double a = 1.0, b = k, c = n + l;
    for (int q = 1; q <= k; q++) {
        for (int i = 0; i < nm; i++) p[i] = 1.0 + a / b * p[i] / c * w[i];
        a = a + 1.0; b = b - 1.0; c = c - 1.0;
    }
    for (int i = 0; i < nm; i++) {
        double mw = -w[i], pw = mw;
        for (int q = 1; q < l + 1; q++) pw = pw * mw;
        vh[i] = factor * p[i] * exp(w[i] / 2.0) * pw;
    }
    free(w); free(p);
}

/* bhwf.f90:2  hydrogenic (n,l) orbital with charge z in the B-spline basis */
int orc_bhwf(const orc_basis *b, int n, int l, double z, double *coef)
{
    int ks = b->ks, ns = b->ns, nv = b->nv;
    double *yr = (double *)malloc(sizeof(double) * nv * ks);
    for (int m = 0; m < ks; m++) {
        vhwf(n, l, z, nv, &b->gr[(size_t)nv * m], &yr[(size_t)nv * m]);
        for (int iv = 0; iv < nv; iv++) yr[iv + (size_t)nv * m] = yr[iv + (size_t)nv * m] * GRW(b, iv, m);
    }
    /* vinty.f90:2 */
    for (int i = 0; i < ns; i++) coef[i] = 0.0;
    for (int ith = 0; ith < ks; ith++)
        for (int iv = 0; iv < nv; iv++)
            for (int m = 0; m < ks; m++)
                coef[iv + ith] = coef[iv + ith] + yr[iv + (size_t)nv * m] * BSP(b, iv, m, ith);
    free(yr);
    /* zfacsb (bhwf.f90:73): full overlap with rows/cols 0..l replaced by identity */
    double *a = (double *)calloc((size_t)ns * ns, sizeof(double));
    for (int jc = 0; jc < ks; jc++)
        for (int i = ks - 1 - jc; i < ns; i++) {
            int j = i + jc - ks + 1;
            a[i + (size_t)ns * j] = BAND(b->sb, ns, i, jc);
            a[j + (size_t)ns * i] = BAND(b->sb, ns, i, jc);
        }
    for (int i = 0; i <= l && i < ns; i++) {
        for (int j = 0; j < ns; j++) { a[i + (size_t)ns * j] = 0.0; a[j + (size_t)ns * i] = 0.0; }
        a[i + (size_t)ns * i] = 1.0;
        coef[i] = 0.0;
    }
    int info = chol_solve(ns, a, coef);
    free(a);
    return info;
}

/* ------------------------------------------------------------------------ */
/* moments.f90:2,76                                                          */
/* ------------------------------------------------------------------------ */
static void moment1(const orc_basis *b, int iv, int k, double *rv, char sym, char dir)
{
    int ks = b->ks;
    double gw[MAXKS];
    for (int m = 0; m < ks; m++) {
        gw[m] = GRW(b, iv, m);
        if (k > 0) { double g = GR(b, iv, m), p = g; for (int q = 1; q < k; q++) p *= g; gw[m] = GRW(b, iv, m) * p; }
        if (k < 0) { double g = GRM(b, iv, m), p = g; for (int q = 1; q < -k; q++) p *= g; gw[m] = GRW(b, iv, m) * p; }
    }
    int ii = 0;
    for (int i = 0; i < ks; i++) {
        int j0 = (sym == 's') ? i : 0;
        for (int j = j0; j < ks; j++) {
            double s = 0.0;
            for (int m = 0; m < ks; m++) {
                double bj = (dir == 'b' ? BSP(b, iv, m, j) : BSQ(b, iv, m, j)) * gw[m];
                s = s + BSP(b, iv, m, i) * bj;
            }
            rv[ii++] = s;
        }
    }
}

/* rkm: (jk, nv) with jk = ks(ks+1)/2 ('s') or ks*ks ('n') */
void orc_moments(const orc_basis *b, int k, double *rkm, char sym, char dir)
{
    int ks = b->ks, nv = b->nv, ml = b->ml, me = b->me;
    int jk = (sym == 'n') ? ks * ks : ks * (ks + 1) / 2;
    double rv[MAXKS * MAXKS];
    if (me == 0) {
        for (int iv = 0; iv < nv; iv++) {
            moment1(b, iv, k, rv, sym, dir);
            memcpy(&rkm[(size_t)jk * iv], rv, sizeof(double) * jk);
        }
        return;
    }
    /* 1-based intervals 1..ml+ks-1 computed, ml+ks..ml+me-ks+2 scaled, rest computed */
    for (int iv = 1; iv <= ml + ks - 1 && iv <= nv; iv++) {
        moment1(b, iv - 1, k, rv, sym, dir);
        memcpy(&rkm[(size_t)jk * (iv - 1)], rv, sizeof(double) * jk);
    }
    double q = 1.0 + b->h, hp = 1.0;
    if (k >= 0) { for (int i = 0; i < k; i++) hp *= q; }
    else { double p = 1.0; for (int i = 0; i < -k; i++) p *= q; hp = 1.0 / p; }
    if (dir == 'b') hp = hp * q;
    for (int iv = ml + ks; iv <= ml + me - ks + 2; iv++)
        for (int i = 0; i < jk; i++)
            rkm[i + (size_t)jk * (iv - 1)] = rkm[i + (size_t)jk * (iv - 2)] * hp;
    for (int iv = ml + me - ks + 3; iv <= nv; iv++) {
        if (iv < 1) continue;
        moment1(b, iv - 1, k, rv, sym, dir);
        memcpy(&rkm[(size_t)jk * (iv - 1)], rv, sizeof(double) * jk);
    }
}

/* ------------------------------------------------------------------------ */
/* rk_moments.f90:105 rk_triang -- diagonal cell iv (0-based), rkd (ik,ik)   */
/* ------------------------------------------------------------------------ */
void orc_rk_triang(const orc_basis *b, int k, int iv, double *rkd_iv)
{
    int ks = b->ks;
    int ik = ks * (ks + 1) / 2;
    int left = iv + ks - 1;
    double xbase = b->t[left];
    double gx[MAXKS], gw[MAXKS], bt[MAXKS * MAXKS], db[MAXKS];
    double *INT = (double *)malloc(sizeof(double) * ks * ks * ks);
    for (int m = 0; m < ks; m++) {
        double span = GR(b, iv, m) - xbase;
        for (int i = 0; i < ks; i++) gx[i] = span * b->gx[i] + xbase;
        for (int i = 0; i < ks; i++) {
            orc_bsplvd(b->t, ks, gx[i], left, 1, db);
            for (int j = 0; j < ks; j++) bt[i + ks * j] = db[j];
        }
        for (int i = 0; i < ks; i++) gw[i] = span * b->gw[i];
        for (int i = 0; i < ks; i++) {
            if (k > 1) { double p = gx[i]; for (int q = 1; q < k; q++) p *= gx[i]; gx[i] = gw[i] * p; }
            else if (k == 1) gx[i] = gw[i] * gx[i];
            else gx[i] = gw[i];
        }
        for (int j = 0; j < ks; j++) {
            double tmp[MAXKS];
            for (int i = 0; i < ks; i++) tmp[i] = gx[i] * bt[i + ks * j];
            for (int jp = j; jp < ks; jp++) {
                double s = 0.0;
                for (int i = 0; i < ks; i++) s = s + tmp[i] * bt[i + ks * jp];
                INT[j + ks * (jp + ks * m)] = s;
            }
        }
    }
    double g2[MAXKS];
    for (int m = 0; m < ks; m++) {
        double g = GRM(b, iv, m), p = g;
        if (k != 0) { for (int q = 1; q < k + 1; q++) p *= g; g2[m] = GRW(b, iv, m) * p; }
        else g2[m] = GRW(b, iv, m) * GRM(b, iv, m);
    }
    double *a = (double *)malloc(sizeof(double) * ik * ik);
    int ii = 0;
    for (int i = 0; i < ks; i++)
        for (int ip = i; ip < ks; ip++) {
            double bi[MAXKS];
            for (int m = 0; m < ks; m++) bi[m] = BSP(b, iv, m, i) * BSP(b, iv, m, ip) * g2[m];
            int jj = 0;
            for (int j = 0; j < ks; j++)
                for (int jp = j; jp < ks; jp++) {
                    double s = 0.0;
                    for (int m = 0; m < ks; m++) s = s + bi[m] * INT[j + ks * (jp + ks * m)];
                    a[ii + ik * jj] = s;
                    jj++;
                }
            ii++;
        }
    for (int c = 0; c < ik; c++)
        for (int r = 0; r < ik; r++)
            rkd_iv[r + ik * c] = a[r + ik * c] + a[c + ik * r];
    free(a);
    free(INT);
}

/* rk_moments.f90:2 -- rkd1,rkd2: (ik,nv); rkd: (ik,ik,nv) */
void orc_rk_moments(const orc_basis *b, int k, double *rkd1, double *rkd2, double *rkd)
{
    int ks = b->ks, nv = b->nv, ml = b->ml, me = b->me;
    int ik = ks * (ks + 1) / 2;
    orc_moments(b, k, rkd1, 's', 'b');
    orc_moments(b, -(k + 1), rkd2, 's', 'b');
    size_t cell = (size_t)ik * ik;
    if (me == 0) {
        for (int iv = 0; iv < nv; iv++) orc_rk_triang(b, k, iv, rkd + cell * iv);
        return;
    }
    for (int iv = 1; iv <= ml + ks - 1 && iv <= nv; iv++) orc_rk_triang(b, k, iv - 1, rkd + cell * (iv - 1));
    double hp = b->h + 1.0;
    for (int iv = ml + ks; iv <= ml + me - ks + 2; iv++)
        for (size_t q = 0; q < cell; q++) rkd[q + cell * (iv - 1)] = rkd[q + cell * (iv - 2)] * hp;
    for (int iv = ml + me - ks + 3; iv <= nv; iv++)
        if (iv >= 1) orc_rk_triang(b, k, iv - 1, rkd + cell * (iv - 1));
}

/* mrk_cell.f90:2 -- rkb (ns,ns,ldp,ldp), zeroed then accumulated */
void orc_mrk_cell_from(const orc_basis *b, const double *rkd1, const double *rkd2,
                       const double *rkd, double *rkb, int ldp)
{
    int ks = b->ks, ns = b->ns, nv = b->nv;
    int ik = ks * (ks + 1) / 2;
    size_t nn = (size_t)ns * ns;
    memset(rkb, 0, sizeof(double) * nn * ldp * ldp);
    for (int jv = 0; jv < nv; jv++) {
        int jj = 0;
        for (int jh = 0; jh < ks; jh++) {
            int j = jv + jh;
            for (int jhp = jh; jhp < ks; jhp++) {
                int jp = jhp - jh;
                for (int iv = 0; iv < nv; iv++) {
                    int ii = 0;
                    for (int ih = 0; ih < ks; ih++) {
                        int i = iv + ih;
                        for (int ihp = ih; ihp < ks; ihp++) {
                            int ip = ihp - ih;
                            double c;
                            if (iv < jv) c = rkd1[ii + (size_t)ik * iv] * rkd2[jj + (size_t)ik * jv];
                            else if (iv > jv) c = rkd1[jj + (size_t)ik * jv] * rkd2[ii + (size_t)ik * iv];
                            else c = rkd[ii + (size_t)ik * (jj + (size_t)ik * iv)];
                            size_t o = i + (size_t)ns * j + nn * (ip + (size_t)ldp * jp);
                            rkb[o] = rkb[o] + c;
                            ii++;
                        }
                    }
                }
                jj++;
            }
        }
    }
}

void orc_mrk_cell(const orc_basis *b, int k, double *rkb, int ldp)
{
    int ks = b->ks, nv = b->nv;
    int ik = ks * (ks + 1) / 2;
    double *rkd1 = (double *)malloc(sizeof(double) * ik * nv);
    double *rkd2 = (double *)malloc(sizeof(double) * ik * nv);
    double *rkd = (double *)malloc(sizeof(double) * ik * ik * nv);
    orc_rk_moments(b, k, rkd1, rkd2, rkd);
    orc_mrk_cell_from(b, rkd1, rkd2, rkd, rkb, ldp);
    free(rkd1); free(rkd2); free(rkd);
}

/* ------------------------------------------------------------------------ */
/* density.f90:2                                                            */
/* ------------------------------------------------------------------------ */
void orc_density(int ns, int ks, double *d, const double *p1, const double *p2, char type)
{
    if (type == 's') {
        memset(d, 0, sizeof(double) * ns * ks);
        for (int i = 0; i < ns; i++) d[i] = p1[i] * p2[i];
        for (int j = 1; j < ks; j++)
            for (int i = 0; i < ns - j; i++)
                d[i + (size_t)ns * j] = p1[i] * p2[i + j] + p1[i + j] * p2[i];
    } else if (type == 'n') {
        memset(d, 0, sizeof(double) * ns * (2 * ks - 1));
        for (int j = 1; j <= 2 * ks - 1; j++) {
            int imin = 1 > 1 + ks - j ? 1 : 1 + ks - j;
            int imax = ns < ns + ks - j ? ns : ns + ks - j;
            for (int i = imin; i <= imax; i++)
                d[(i - 1) + (size_t)ns * (j - 1)] = p1[i - 1] * p2[i + j - ks - 1];
        }
    } else {
        for (int i = 0; i < ns; i++)
            for (int j = 0; j < ns; j++) d[i + (size_t)ns * j] = p1[i] * p2[j];
    }
}

/* ------------------------------------------------------------------------ */
/* convol.f90:2 -- literal restatement, 1-based loop variables               */
/* ------------------------------------------------------------------------ */
int orc_convol(int ns, int ks, double *a, const double *d, const double *rkb, int ldp,
               int icase, char si, char sj)
{
    size_t nn = (size_t)ns * ns;
#define R(i, j, ip, jp) rkb[((i) - 1) + (size_t)ns * ((j) - 1) + nn * (((ip) - 1) + (size_t)ldp * ((jp) - 1))]
#define Dm(i, j) d[((i) - 1) + (size_t)ns * ((j) - 1)]
#define Am(i, j) a[((i) - 1) + (size_t)ns * ((j) - 1)]
#define MAX(x, y) ((x) > (y) ? (x) : (y))
#define MIN(x, y) ((x) < (y) ? (x) : (y))
    int k2 = ks + ks - 1;
    if (icase > 2) memset(a, 0, sizeof(double) * nn);
    if (si == 's' && sj == 's' && icase == 1) {
        for (int ip = 1; ip <= ks; ip++)
            for (int i = 1; i <= ns - ip + 1; i++) {
                double c = 0.0;
                for (int jp = 1; jp <= ks; jp++)
                    for (int j = 1; j <= ns - jp + 1; j++) c = c + Dm(j, jp) * R(i, j, ip, jp);
                Am(i, ip) = c;
            }
    } else if (si == 's' && sj == 's' && icase == 2) {
        for (int ip = 1; ip <= ks; ip++)
            for (int i = 1; i <= ns - ip + 1; i++) {
                double c = 0.0;
                for (int jp = 1; jp <= ks; jp++)
                    for (int j = 1; j <= ns - jp + 1; j++) c = c + Dm(j, jp) * R(j, i, jp, ip);
                Am(i, ip) = c;
            }
    } else if (si == 'n' && sj == 'n' && icase == 1) {
        for (int ip = 1; ip <= k2; ip++) {
            int imin = MAX(1, 1 + ks - ip), imax = MIN(ns, ns + ks - ip);
            for (int i = imin; i <= imax; i++) {
                double c = 0.0;
                for (int jp = 1; jp <= k2; jp++) {
                    int jmin = MAX(1, 1 + ks - jp), jmax = MIN(ns, ns + ks - jp);
                    for (int j = jmin; j <= jmax; j++) c = c + Dm(j, jp) * R(i, j, ip, jp);
                }
                Am(i, ip) = c;
            }
        }
    } else if (si == 'n' && sj == 'n' && icase == 2) {
        for (int ip = 1; ip <= k2; ip++) {
            int imin = MAX(1, 1 + ks - ip), imax = MIN(ns, ns + ks - ip);
            for (int i = imin; i <= imax; i++) {
                double c = 0.0;
                for (int jp = 1; jp <= k2; jp++) {
                    int jmin = MAX(1, 1 + ks - jp), jmax = MIN(ns, ns + ks - jp);
                    for (int j = jmin; j <= jmax; j++) c = c + Dm(j, jp) * R(j, i, jp, ip);
                }
                Am(i, ip) = c;
            }
        }
    } else if (si == 'n' && sj == 's' && icase == 1) {
        for (int ip = 1; ip <= k2; ip++) {
            int imin = MAX(1, 1 + ks - ip), imax = MIN(ns, ns + ks - ip);
            for (int i = imin; i <= imax; i++) {
                double c = 0.0;
                for (int jp = 1; jp <= ks; jp++)
                    for (int j = 1; j <= ns - jp + 1; j++) c = c + Dm(j, jp) * R(i, j, ip, jp);
                Am(i, ip) = c;
            }
        }
    } else if (si == 'n' && sj == 's' && icase == 2) {
        for (int jp = 1; jp <= ks; jp++)
            for (int j = 1; j <= ns - jp + 1; j++) {
                double c = 0.0;
                for (int ip = 1; ip <= k2; ip++) {
                    int imin = MAX(1, 1 + ks - ip), imax = MIN(ns, ns + ks - ip);
                    for (int i = imin; i <= imax; i++) c = c + Dm(i, ip) * R(i, j, ip, jp);
                }
                Am(j, jp) = c;
            }
    } else if (si == 's' && sj == 'n' && icase == 2) {
        for (int jp = 1; jp <= k2; jp++) {
            int jmin = MAX(1, 1 + ks - jp), jmax = MIN(ns, ns + ks - jp);
            for (int j = jmin; j <= jmax; j++) {
                double c = 0.0;
                for (int ip = 1; ip <= ks; ip++)
                    for (int i = 1; i <= ns - ip + 1; i++) c = c + Dm(i, ip) * R(i, j, ip, jp);
                Am(j, jp) = c;
            }
        }
    } else if (si == 's' && sj == 'n' && icase == 1) {
        for (int ip = 1; ip <= ks; ip++)
            for (int i = 1; i <= ns - ip + 1; i++) {
                double c = 0.0;
                for (int jp = 1; jp <= k2; jp++) {
                    int jmin = MAX(1, 1 + ks - jp), jmax = MIN(ns, ns + ks - jp);
                    for (int j = jmin; j <= jmax; j++) c = c + Dm(j, jp) * R(i, j, ip, jp);
                }
                Am(i, ip) = c;
            }
    } else if (si == 's' && sj == 's' && icase == 3) {
        for (int jp = 1; jp <= ks; jp++)
            for (int j = 1; j <= ns - jp + 1; j++) {
                int jj = j + jp - 1;
                for (int ip = 1; ip <= ks; ip++)
                    for (int i = 1; i <= ns - ip + 1; i++) {
                        int ii = i + ip - 1;
                        double c = R(i, j, ip, jp);
                        Am(i, jj) = Am(i, jj) + c * Dm(ii, j);
                        if (ip > 1) Am(ii, jj) = Am(ii, jj) + c * Dm(i, j);
                        if (jp > 1) Am(i, j) = Am(i, j) + c * Dm(ii, jj);
                        if (ip > 1 && jp > 1) Am(ii, j) = Am(ii, j) + c * Dm(i, jj);
                    }
            }
    } else if (si == 's' && sj == 's' && icase == 4) {
        for (int jp = 1; jp <= ks; jp++)
            for (int j = 1; j <= ns - jp + 1; j++) {
                int jj = j + jp - 1;
                for (int ip = 1; ip <= ks; ip++)
                    for (int i = 1; i <= ns - ip + 1; i++) {
                        int ii = i + ip - 1;
                        double c = R(i, j, ip, jp);
                        Am(ii, j) = Am(ii, j) + c * Dm(i, jj);
                        if (ip > 1) Am(i, j) = Am(i, j) + c * Dm(ii, jj);
                        if (jp > 1) Am(ii, jj) = Am(ii, jj) + c * Dm(i, j);
                        if (ip > 1 && jp > 1) Am(i, jj) = Am(i, jj) + c * Dm(ii, j);
                    }
            }
    } else if (si == 'n' && sj == 'n' && icase == 3) {
        for (int jp = 1; jp <= k2; jp++) {
            int jmin = MAX(1, 1 + ks - jp), jmax = MIN(ns, ns + ks - jp);
            for (int j = jmin; j <= jmax; j++) {
                int jj = j + jp - ks;
                for (int ip = 1; ip <= k2; ip++) {
                    int imin = MAX(1, 1 + ks - ip), imax = MIN(ns, ns + ks - ip);
                    for (int i = imin; i <= imax; i++) {
                        int ii = i + ip - ks;
                        Am(i, jj) = Am(i, jj) + R(i, j, ip, jp) * Dm(ii, j);
                    }
                }
            }
        }
    } else if (si == 'n' && sj == 'n' && icase == 4) {
        for (int jp = 1; jp <= k2; jp++) {
            int jmin = MAX(1, 1 + ks - jp), jmax = MIN(ns, ns + ks - jp);
            for (int j = jmin; j <= jmax; j++) {
                int jj = j + jp - ks;
                for (int ip = 1; ip <= k2; ip++) {
                    int imin = MAX(1, 1 + ks - ip), imax = MIN(ns, ns + ks - ip);
                    for (int i = imin; i <= imax; i++) {
                        int ii = i + ip - ks;
                        Am(ii, j) = Am(ii, j) + R(i, j, ip, jp) * Dm(i, jj);
                    }
                }
            }
        }
    } else if (si == 'n' && sj == 's' && icase == 3) {
        for (int jp = 1; jp <= ks; jp++)
            for (int j = 1; j <= ns - jp + 1; j++) {
                int jj = j + jp - 1;
                for (int ip = 1; ip <= k2; ip++) {
                    int imin = MAX(1, 1 + ks - ip), imax = MIN(ns, ns + ks - ip);
                    for (int i = imin; i <= imax; i++) {
                        int ii = i + ip - ks;
                        Am(i, jj) = Am(i, jj) + R(i, j, ip, jp) * Dm(ii, j);
                        if (jp > 1) Am(i, j) = Am(i, j) + R(i, j, ip, jp) * Dm(ii, jj);
                    }
                }
            }
    } else if (si == 'n' && sj == 's' && icase == 4) {
        for (int jp = 1; jp <= ks; jp++)
            for (int j = 1; j <= ns - jp + 1; j++) {
                int jj = j + jp - 1;
                for (int ip = 1; ip <= k2; ip++) {
                    int imin = MAX(1, 1 + ks - ip), imax = MIN(ns, ns + ks - ip);
                    for (int i = imin; i <= imax; i++) {
                        int ii = i + ip - ks;
                        Am(ii, j) = Am(ii, j) + R(i, j, ip, jp) * Dm(i, jj);
                        if (jp > 1) Am(ii, jj) = Am(ii, jj) + R(i, j, ip, jp) * Dm(i, j);
                    }
                }
            }
    } else if (si == 's' && sj == 'n' && icase == 3) {
        for (int jp = 1; jp <= k2; jp++) {
            int jmin = MAX(1, 1 + ks - jp), jmax = MIN(ns, ns + ks - jp);
            for (int j = jmin; j <= jmax; j++) {
                int jj = j + jp - ks;
                for (int ip = 1; ip <= ks; ip++)
                    for (int i = 1; i <= ns - ip + 1; i++) {
                        int ii = i + ip - 1;
                        Am(i, jj) = Am(i, jj) + R(i, j, ip, jp) * Dm(ii, j);
                        if (ip > 1) Am(ii, jj) = Am(ii, jj) + R(i, j, ip, jp) * Dm(i, j);
                    }
            }
        }
    } else if (si == 's' && sj == 'n' && icase == 4) {
        for (int jp = 1; jp <= k2; jp++) {
            int jmin = MAX(1, 1 + ks - jp), jmax = MIN(ns, ns + ks - jp);
            for (int j = jmin; j <= jmax; j++) {
                int jj = j + jp - ks;
                for (int ip = 1; ip <= ks; ip++)
                    for (int i = 1; i <= ns - ip + 1; i++) {
                        int ii = i + ip - 1;
                        Am(ii, j) = Am(ii, j) + R(i, j, ip, jp) * Dm(i, jj);
                        if (ip > 1) Am(i, j) = Am(i, j) + R(i, j, ip, jp) * Dm(ii, jj);
                    }
            }
        }
    } else {
        return -1;   /* convol.f90: Stop ' CONVOL:  unknown case ' */
    }
    return 0;
#undef R
#undef Dm
#undef Am
}

/* sum_amb.f90:2 */
double orc_sum_amb(int ns, int ks, const double *a, const double *b, char sym)
{
    double x = 0.0;
    if (sym == 'x') {
        for (int i = 0; i < ns; i++)
            for (int j = 0; j < ns; j++) x = x + a[i + (size_t)ns * j] * b[i + (size_t)ns * j];
    } else if (sym == 's') {
        for (int j = 1; j <= ks; j++)
            for (int i = 1; i <= ns - j + 1; i++) x = x + a[(i - 1) + (size_t)ns * (j - 1)] * b[(i - 1) + (size_t)ns * (j - 1)];
    } else if (sym == 'l') {
        for (int j = 1; j <= ks; j++)
            for (int i = ks + 1 - j; i <= ns; i++) x = x + a[(i - 1) + (size_t)ns * (j - 1)] * b[(i - 1) + (size_t)ns * (j - 1)];
    } else if (sym == 'n') {
        for (int j = 1; j <= ks + ks - 1; j++) {
            int imin = MAX(1, 1 + ks - j), imax = MIN(ns, ns + ks - j);
            for (int i = imin; i <= imax; i++) x = x + a[(i - 1) + (size_t)ns * (j - 1)] * b[(i - 1) + (size_t)ns * (j - 1)];
        }
    } else return NAN;
    return x;
}

/* bav.f90:2 */
void orc_bav(int ns, int ks, const double *bm, const double *v, double *y, char type, char side)
{
    if (type == 's') {
        for (int i = 0; i < ns; i++) y[i] = bm[i] * v[i];
        for (int ip = 2; ip <= ks; ip++)
            for (int i = 1; i <= ns - ip + 1; i++) {
                int j = i + ip - 1;
                double c = bm[(i - 1) + (size_t)ns * (ip - 1)];
                y[i - 1] = y[i - 1] + c * v[j - 1];
                y[j - 1] = y[j - 1] + c * v[i - 1];
            }
    } else if (type == 'n') {
        for (int i = 0; i < ns; i++) y[i] = 0.0;
        for (int ip = 1; ip <= ks + ks - 1; ip++) {
            int imin = MAX(1, 1 + ks - ip), imax = MIN(ns, ns + ks - ip);
            for (int i = imin; i <= imax; i++) {
                int j = i + ip - ks;
                double c = bm[(i - 1) + (size_t)ns * (ip - 1)];
                if (side == 'r') y[i - 1] = y[i - 1] + c * v[j - 1];
                else y[j - 1] = y[j - 1] + c * v[i - 1];
            }
        }
    }
}

/* bvmv.f90:2 */
double orc_bvmv(int n, int k, const double *ar, char type, const double *x, const double *y)
{
    double s = 0.0;
#define AR(i, j) ar[((i) - 1) + (size_t)n * ((j) - 1)]
    if (type != 'g') {
        for (int jp = 1; jp <= k - 1; jp++)
            for (int i = k + 1 - jp; i <= n; i++) {
                int j = i + jp - k;
                s = s + AR(i, jp) * (x[i - 1] * y[j - 1] + x[j - 1] * y[i - 1]);
            }
        if (type == 'a') s = s + x[n - 2] * y[n - 1] * (AR(1, 1) - AR(n, k - 1));
    } else {
        for (int jp = 1; jp <= k - 1; jp++)
            for (int i = k - jp + 1; i <= n; i++) {
                int j = i + jp - k, kp = 2 * k - jp;
                s = s + AR(i, jp) * x[i - 1] * y[j - 1];
                s = s + AR(j, kp) * x[j - 1] * y[i - 1];
            }
    }
    double c = 0.0;
    for (int i = 1; i <= n; i++) c = c + AR(i, k) * x[i - 1] * y[i - 1];
    s = s + c;
#undef AR
    return s;
}

/* quadr.f90:2  <p1 | r^m | p2> */
double orc_quadr(const orc_basis *b, const double *p1, const double *p2, int m)
{
    int ns = b->ns, ks = b->ks;
    if (m == 1) return orc_bvmv(ns, ks, b->r1, 's', p1, p2);
    if (m == 0) return orc_bvmv(ns, ks, b->sb, 's', p1, p2);
    if (m == -1) return orc_bvmv(ns, ks, b->rm1, 's', p1, p2);
    if (m == -2) return orc_bvmv(ns, ks, b->rm2, 's', p1, p2);
    double *rm = (double *)malloc(sizeof(double) * ns * ks);
    orc_mrm(b, m, rm);
    double v = orc_bvmv(ns, ks, rm, 's', p1, p2);
    free(rm);
    return v;
}

/* rk.f90:2  R^k(i1,j1;i2,j2) from a filled rkb (ldp) */
double orc_rk(int ns, int ks, const double *rkb, int ldp, const double *pi1, const double *pj1,
              const double *pi2, const double *pj2)
{
    double *a = (double *)malloc(sizeof(double) * ns * ks), *bb = (double *)malloc(sizeof(double) * ns * ks);
    size_t nn = (size_t)ns * ns;
    orc_density(ns, ks, a, pi1, pi2, 's');
    orc_density(ns, ks, bb, pj1, pj2, 's');
    double rk = 0.0;
    for (int ip = 1; ip <= ks; ip++)
        for (int i = 1; i <= ns - ip + 1; i++) {
            double rkj = 0.0;
            for (int jp = 1; jp <= ks; jp++)
                for (int j = 1; j <= ns - jp + 1; j++)
                    rkj = rkj + bb[(j - 1) + (size_t)ns * (jp - 1)] *
                                rkb[(j - 1) + (size_t)ns * (i - 1) + nn * ((jp - 1) + (size_t)ldp * (ip - 1))];
            rk = rk + a[(i - 1) + (size_t)ns * (ip - 1)] * rkj;
        }
    free(a); free(bb);
    return rk;
}

/* int_de.f90:2 for Rk (int=5): sym_i = sym_j = 's'.  x must hold ns*ns. */
static void int_de_rk(int ns, int ks, const double *rkb, int ldp, const double *p1, const double *p2,
                      double *x, int icase, char *sym_x)
{
    double *d = (double *)malloc(sizeof(double) * ns * ns);
    char sym_d = (icase <= 2) ? 's' : 'x';
    orc_density(ns, ks, d, p1, p2, sym_d);
    orc_convol(ns, ks, x, d, rkb, ldp, icase, 's', 's');
    *sym_x = (icase <= 2) ? 's' : 'x';
    free(d);
}

/* test_bs.f90:2177 rkd (fine = 1) */
double orc_rkd(int ns, int ks, const double *rkb, int ldp, const double *pi1, const double *pj1,
               const double *pi2, const double *pj2)
{
    double *a = (double *)malloc(sizeof(double) * ns * ns), *bb = (double *)malloc(sizeof(double) * ns * ns);
    char sym;
    double r = 0.0;
    int_de_rk(ns, ks, rkb, ldp, pi1, pi2, a, 2, &sym);
    orc_density(ns, ks, bb, pj1, pj2, sym);
    r = r + orc_sum_amb(ns, ks, a, bb, sym);
    int_de_rk(ns, ks, rkb, ldp, pj1, pj2, a, 1, &sym);
    orc_density(ns, ks, bb, pi1, pi2, sym);
    r = r + orc_sum_amb(ns, ks, a, bb, sym);
    free(a); free(bb);
    return r * 1.0 / 2;
}

/* test_bs.f90:2216 rke */
double orc_rke(int ns, int ks, const double *rkb, int ldp, const double *pi1, const double *pj1,
               const double *pi2, const double *pj2)
{
    double *a = (double *)malloc(sizeof(double) * ns * ns), *bb = (double *)malloc(sizeof(double) * ns * ns);
    char sym;
    double r = 0.0;
    int_de_rk(ns, ks, rkb, ldp, pi2, pj1, a, 3, &sym);
    orc_density(ns, ks, bb, pi1, pj2, sym);
    r = r + orc_sum_amb(ns, ks, a, bb, sym);
    int_de_rk(ns, ks, rkb, ldp, pi1, pj2, a, 4, &sym);
    orc_density(ns, ks, bb, pi2, pj1, sym);
    r = r + orc_sum_amb(ns, ks, a, bb, sym);
    free(a); free(bb);
    return r / 2;
}

/* test_bs.f90:1091 rkv with INT_v (int_v.f90) */
double orc_rkv(int ns, int ks, const double *rkb, int ldp, const double *pi1, const double *pj1,
               const double *pi2, const double *pj2)
{
    double *x = (double *)malloc(sizeof(double) * ns * ns), *v = (double *)malloc(sizeof(double) * ns);
    char sym;
    double r = 0.0, s;
    /* icase 1 */
    int_de_rk(ns, ks, rkb, ldp, pj1, pj2, x, 1, &sym);
    orc_bav(ns, ks, x, pi2, v, sym, 'r');
    s = 0.0; for (int i = 0; i < ns; i++) s = s + v[i] * pi1[i]; r = r + s;
    /* icase 2 */
    int_de_rk(ns, ks, rkb, ldp, pi1, pi2, x, 2, &sym);
    orc_bav(ns, ks, x, pj2, v, sym, 'r');
    s = 0.0; for (int i = 0; i < ns; i++) s = s + v[i] * pj1[i]; r = r + s;
    /* icase 3 */
    int_de_rk(ns, ks, rkb, ldp, pj1, pj2, x, 1, &sym);
    orc_bav(ns, ks, x, pi1, v, sym, 'l');
    s = 0.0; for (int i = 0; i < ns; i++) s = s + v[i] * pi2[i]; r = r + s;
    /* icase 4 */
    int_de_rk(ns, ks, rkb, ldp, pi1, pi2, x, 2, &sym);
    orc_bav(ns, ks, x, pj1, v, sym, 'l');
    s = 0.0; for (int i = 0; i < ns; i++) s = s + v[i] * pj2[i]; r = r + s;
    free(x); free(v);
    return r * 1.0 / 4;
}

/* ------------------------------------------------------------------------ */
/* one-electron operator: l_core.f90:174 INT_core with no closed shells     */
/* hl_full (ns,ns) = symmetric full matrix of db2 - l(l+1) rm2 + 2z rm1     */
/* with the Bloch correction at the right border.                           */
/* ------------------------------------------------------------------------ */
void orc_hl_full(const orc_basis *b, int l, double z, double *hl_full)
{
    int ns = b->ns, ks = b->ks;
    double *hl = (double *)malloc(sizeof(double) * ns * ks);
    double c1 = (double)(l * (l + 1)), c2 = 2 * z;
    for (size_t q = 0; q < (size_t)ns * ks; q++) hl[q] = b->db2[q] - c1 * b->rm2[q] + c2 * b->rm1[q];
    double cb = b->db2[0] - BAND(b->db2, ns, ns - 1, ks - 2);
    BAND(hl, ns, ns - 1, ks - 2) = BAND(hl, ns, ns - 1, ks - 2) + cb;
    BAND(hl, ns, ns - 1, ks - 1) = BAND(hl, ns, ns - 1, ks - 1) - cb;
    memset(hl_full, 0, sizeof(double) * ns * ns);
    for (int jp = 1; jp <= ks; jp++)
        for (int i = 1 - jp + ks; i <= ns; i++) {
            int j = i + jp - ks;
            hl_full[(i - 1) + (size_t)ns * (j - 1)] = hl_full[(i - 1) + (size_t)ns * (j - 1)] + hl[(i - 1) + (size_t)ns * (jp - 1)];
            hl_full[(j - 1) + (size_t)ns * (i - 1)] = hl_full[(i - 1) + (size_t)ns * (j - 1)];
        }
    free(hl);
}

/* ------------------------------------------------------------------------ */
/* channel-block assembly of one partial wave                               */
/*                                                                          */
/* hcc (ns,ns,nch(nch+1)/2), block ij = i*(i-1)/2 + j (1-based, i >= j).    */
/* Coefficient records, sorted by (k, type, ich, jch):                      */
/*   ck[t] multipole, ctype[t] 0 = direct Rk(i . j .) (jcase 1, 's' density,*/
/*   band result) or 1 = exchange Rk(i . . j) (jcase 3, 'x' density, full   */
/*   result); cich/cjch 1-based channels (cich >= cjch); ca/cb 0-based      */
/*   orbital columns of P; cval the angular coefficient.                    */
/* acf (nch,nch,kmax+1) receives Sum c*<a|r^k|b> of the direct groups.      */
/* The rkb tables for k=0..kmax are given as one (ns,ns,ks,ks,kmax+1) array.*/
/* ------------------------------------------------------------------------ */
static void update_hx(int nch, int ns, int ks, double *hcc, int ich, int jch, const double *d, char sym, double *x)
{
    (void)nch;
    memset(x, 0, sizeof(double) * ns * ns);
    if (sym == 's') {
        for (int ith = 1; ith <= ks; ith++)
            for (int i = 1; i <= ns - ith + 1; i++) {
                int j = i + ith - 1;
                x[(i - 1) + (size_t)ns * (j - 1)] = d[(i - 1) + (size_t)ns * (ith - 1)];
                x[(j - 1) + (size_t)ns * (i - 1)] = d[(i - 1) + (size_t)ns * (ith - 1)];
            }
    } else {
        memcpy(x, d, sizeof(double) * ns * ns);
    }
    int i = ich > jch ? ich : jch, j = ich > jch ? jch : ich;
    size_t ij = (size_t)i * (i - 1) / 2 + j - 1;
    double *blk = hcc + ij * ns * ns;
    if (ich >= jch) {
        for (size_t q = 0; q < (size_t)ns * ns; q++) blk[q] = blk[q] + x[q];
    } else {
        for (int c = 0; c < ns; c++)
            for (int r = 0; r < ns; r++) blk[r + (size_t)ns * c] = blk[r + (size_t)ns * c] + x[c + (size_t)ns * r];
    }
}

static void update_hl(int ns, int ks, double *hcc, int ich, int jch, const double *d, double c)
{
    int i0 = ich > jch ? ich : jch, j0 = ich > jch ? jch : ich;
    size_t ij = (size_t)i0 * (i0 - 1) / 2 + j0 - 1;
    double *blk = hcc + ij * ns * ns;
    for (int ith = 1; ith <= ks; ith++)
        for (int i = ks + 1 - ith; i <= ns; i++) {
            int j = i + ith - ks;
            double s = c * d[(i - 1) + (size_t)ns * (ith - 1)];
            blk[(i - 1) + (size_t)ns * (j - 1)] = blk[(i - 1) + (size_t)ns * (j - 1)] + s;
            if (i != j) blk[(j - 1) + (size_t)ns * (i - 1)] = blk[(j - 1) + (size_t)ns * (i - 1)] + s;
        }
}

int orc_assemble(const orc_basis *b, double z, int nch, const int *lch, const double *ech,
                 int norb, const double *P, int kmax, const double *rkb_all,
                 int ncoef, const int *ck, const int *ctype, const int *cich, const int *cjch,
                 const int *ca, const int *cb, const double *cval,
                 double *hcc, double *scc, double *acf)
{
    int ns = b->ns, ks = b->ks;
    size_t nn = (size_t)ns * ns;
    size_t nblk = (size_t)nch * (nch + 1) / 2;
    (void)norb;
    memset(hcc, 0, sizeof(double) * nn * nblk);
    if (scc) {
        memset(scc, 0, sizeof(double) * nn * nblk);
        for (int ich = 1; ich <= nch; ich++) update_hl(ns, ks, scc, ich, ich, b->sb, 1.0);
        for (int ich = 1; ich <= nch; ich++) {
            double *blk = scc + ((size_t)ich * (ich + 1) / 2 - 1) * nn;
            for (int i = 1; i <= ns; i++)
                for (int j = 1; j <= i; j++) {
                    double c = blk[(i - 1) + (size_t)ns * (j - 1)] + blk[(j - 1) + (size_t)ns * (i - 1)];
                    blk[(i - 1) + (size_t)ns * (j - 1)] = c / 2.0;
                    blk[(j - 1) + (size_t)ns * (i - 1)] = c / 2.0;
                }
        }
    }
    if (acf) memset(acf, 0, sizeof(double) * nch * nch * (kmax + 1));
    double *x = (double *)malloc(sizeof(double) * nn);
    double *xx = (double *)malloc(sizeof(double) * nn);
    double *dd = (double *)malloc(sizeof(double) * nn);
    double *hl = (double *)malloc(sizeof(double) * nn);
    /* L-integrals: L_data Case(6..9) with C = -1/2 on each channel's diagonal block */
    for (int ich = 1; ich <= nch; ich++) {
        orc_hl_full(b, lch[ich - 1], z, hl);
        for (size_t q = 0; q < nn; q++) xx[q] = -0.5 * hl[q];
        update_hx(nch, ns, ks, hcc, ich, ich, xx, 'x', x);
    }
    /* R-integrals: I_data Case(6..9) group loop */
    int t = 0;
    while (t < ncoef) {
        int k = ck[t], ty = ctype[t], ich = cich[t], jch = cjch[t];
        if (k < 0 || k > kmax || ich < 1 || ich > nch || jch < 1 || jch > nch) {
            free(x); free(xx); free(dd); free(hl);
            return -1;
        }
        char sym_d = ty == 0 ? 's' : 'x';
        int jcase = ty == 0 ? 1 : 3;
        memset(xx, 0, sizeof(double) * nn);
        double CA = 0.0;
        int t0 = t;
        while (t < ncoef && ck[t] == k && ctype[t] == ty && cich[t] == ich && cjch[t] == jch) {
            const double *pa = P + (size_t)ns * ca[t], *pb = P + (size_t)ns * cb[t];
            orc_density(ns, ks, dd, pa, pb, sym_d);
            size_t len = (sym_d == 's') ? (size_t)ns * ks : nn;
            for (size_t q = 0; q < len; q++) xx[q] = xx[q] + cval[t] * dd[q];
            if (acf && ty == 0) CA = CA + cval[t] * orc_quadr(b, pa, pb, k);
            t++;
        }
        (void)t0;
        const double *rkb = rkb_all + nn * ks * ks * (size_t)k;
        orc_convol(ns, ks, dd, xx, rkb, ks, jcase, 's', 's');
        update_hx(nch, ns, ks, hcc, ich, jch, dd, ty == 0 ? 's' : 'x', x);
        if (acf && ty == 0) acf[(ich - 1) + (size_t)nch * ((jch - 1) + (size_t)nch * k)] += CA;
    }
    /* target energies: UPDATE_HL(i,i,sb,Etarg-EC) with EC = 0 */
    for (int ich = 1; ich <= nch; ich++) update_hl(ns, ks, hcc, ich, ich, b->sb, ech[ich - 1]);
    /* symmetrise diagonal blocks */
    for (int ich = 1; ich <= nch; ich++) {
        double *blk = hcc + ((size_t)ich * (ich + 1) / 2 - 1) * nn;
        for (int i = 1; i <= ns; i++)
            for (int j = 1; j <= i; j++) {
                double c = blk[(i - 1) + (size_t)ns * (j - 1)] + blk[(j - 1) + (size_t)ns * (i - 1)];
                blk[(i - 1) + (size_t)ns * (j - 1)] = c / 2.0;
                blk[(j - 1) + (size_t)ns * (i - 1)] = c / 2.0;
            }
    }
    free(x); free(xx); free(dd); free(hl);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* BS_ORTH (src/bsr/BSR_MAT3/bs_orth.f90:2-92): orthogonality conditions of  */
/* the channels by Bentley's projection H -> (1 - B zz) H (1 - zz B), zz =  */
/* Sum_j p_j p_j^T over the orbitals listed for the channel (ort_ptr/ort_idx,*/
/* 0-based orbital columns of P), B = full overlap (Full_mat_sym of sb, 'l').*/
/* Channels are processed one after another as in the reference (:38-86).   */
/* ------------------------------------------------------------------------ */
static void matmul_nn(int n, const double *a, const double *b, double *c)
{
    for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++) {
            double s = 0.0;
            for (int k = 0; k < n; k++) s += a[i + (size_t)n * k] * b[k + (size_t)n * j];
            c[i + (size_t)n * j] = s;
        }
}

int orc_bs_orth(int ns, int ks, const double *sb, int nch, const double *P, const int *ort_ptr, const int *ort_idx,
                double *hcc)
{
    size_t nn = (size_t)ns * ns;
    double *B = (double *)calloc(nn, sizeof(double));
    double *zz = (double *)malloc(sizeof(double) * nn);
    double *x = (double *)malloc(sizeof(double) * nn);
    double *y = (double *)malloc(sizeof(double) * nn);
    double *xx = (double *)malloc(sizeof(double) * nn);
    /* Full_mat_sym(ns,ks,sb,bb,'l') */
    for (int jp = 1; jp <= ks; jp++)
        for (int i = ks + 1 - jp; i <= ns; i++) {
            int j = i + jp - ks;
            B[(i - 1) + (size_t)ns * (j - 1)] = sb[(i - 1) + (size_t)ns * (jp - 1)];
            B[(j - 1) + (size_t)ns * (i - 1)] = sb[(i - 1) + (size_t)ns * (jp - 1)];
        }
    for (int ich = 1; ich <= nch; ich++) {
        int nort = ort_ptr[ich] - ort_ptr[ich - 1];
        if (nort == 0) continue;
        memset(zz, 0, sizeof(double) * nn);
        for (int q = ort_ptr[ich - 1]; q < ort_ptr[ich]; q++) {
            const double *z = P + (size_t)ns * ort_idx[q];
            for (int ii = 0; ii < ns; ii++)
                for (int jj = 0; jj < ns; jj++) zz[ii + (size_t)ns * jj] += z[ii] * z[jj];
        }
        matmul_nn(ns, B, zz, x);
        matmul_nn(ns, zz, B, y);
        for (int jch = 1; jch <= nch; jch++) {
            size_t ij;
            double *h;
            if (ich > jch) {
                ij = (size_t)ich * (ich - 1) / 2 + jch - 1;
                h = hcc + ij * nn;
                matmul_nn(ns, x, h, xx);
                for (size_t q = 0; q < nn; q++) h[q] -= xx[q];
            } else if (ich == jch) {
                ij = (size_t)ich * (ich + 1) / 2 - 1;
                h = hcc + ij * nn;
                matmul_nn(ns, x, h, xx);
                for (size_t q = 0; q < nn; q++) h[q] -= xx[q];
                matmul_nn(ns, h, y, xx);
                for (size_t q = 0; q < nn; q++) h[q] -= xx[q];
            } else {
                ij = (size_t)jch * (jch - 1) / 2 + ich - 1;
                h = hcc + ij * nn;
                matmul_nn(ns, h, y, xx);
                for (size_t q = 0; q < nn; q++) h[q] -= xx[q];
            }
        }
    }
    free(B); free(zz); free(x); free(y); free(xx);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* rsol_out (src/bsr/BSR_HD3/rsol_out.f90:20-36): the solutions in the      */
/* B-spline basis v(:,is) = Sum_j a(j,is) bb(:,j) channel by channel and the*/
/* surface amplitudes WMAT(ich,is) = v(ich*ns, is).  bb: (ns, nch*ns), the  */
/* channel eigenbasis with ns columns reserved per channel (ipsol offsets). */
/* ------------------------------------------------------------------------ */
void orc_rsol(int ns, int nch, const int *ipsol, const double *bb, int khm, const double *a, double *v, double *wmat)
{
    int nhm = nch * ns;
    for (int is = 0; is < khm; is++) {
        for (int ich = 0; ich < nch; ich++) {
            for (int r = 0; r < ns; r++) {
                double s = 0.0;
                for (int j = ipsol[ich]; j < ipsol[ich + 1]; j++)
                    s += a[j + (size_t)khm * is] * bb[r + (size_t)ns * ((size_t)ich * ns + (j - ipsol[ich]))];
                if (v) v[(size_t)ich * ns + r + (size_t)nhm * is] = s;
                if (r == ns - 1) wmat[ich + (size_t)nch * is] = s;
            }
        }
    }
}

/* ------------------------------------------------------------------------ */
/* W_OUT weights (w_out.f90:58-76): cval = a(:,is)^2, WT(ich) = SUM(cval over  */
/* the channel's rows), SORTA (ZCOM/sorting_routines.f90:79-97) of |WT| into */
/* iprm, isol = iprm(1).  wt, iprm: (nch, khm); iprm/isol 1-based.           */
/* ------------------------------------------------------------------------ */
void orc_channel_weights(int nch, const int *ipsol, int khm, const double *a, double *wt, int *isol, int *iprm)
{
    int *ipt = (int *)malloc(sizeof(int) * (size_t)nch);
    for (int is = 0; is < khm; is++) {
        const double *col = a + (size_t)khm * is;
        double *w = wt + (size_t)nch * is;
        for (int ich = 0; ich < nch; ich++) {
            double s = 0.0;
            for (int j = ipsol[ich]; j < ipsol[ich + 1]; j++) {
                double cv = col[j] * col[j];
                s = s + cv;
            }
            w[ich] = s;
        }
        for (int i = 0; i < nch; i++) ipt[i] = i;
        for (int i1 = 0; i1 < nch - 1; i1++) {
            int j1 = ipt[i1];
            for (int i2 = i1 + 1; i2 < nch; i2++) {
                int j2 = ipt[i2];
                if (fabs(w[j1]) < fabs(w[j2])) {
                    ipt[i2] = j1;
                    j1 = j2;
                }
            }
            ipt[i1] = j1;
        }
        isol[is] = ipt[0] + 1;
        if (iprm)
            for (int i = 0; i < nch; i++) iprm[i + (size_t)nch * is] = ipt[i] + 1;
    }
    free(ipt);
}

/* ------------------------------------------------------------------------ */
/* Breit-Pauli N^k tables: nk_moments.f90:2-189 (moments k and -(k+3),       */
/* nk_pdiag :56 with the scaling law rkd(iv) = rkd(iv-1)/(1+h), nk_triang    */
/* :105 -- the one-sided diagonal cell r2 < r1, not symmetrised) and         */
/* mnk_cell.f90:2-85 (cells jv <= iv only, times `fine`).                    */
/* ------------------------------------------------------------------------ */
static double ipow(double x, int k)
{
    if (k == 0) return 1.0;
    double p = x;
    for (int q = 1; q < (k > 0 ? k : -k); q++) p *= x;
    return k > 0 ? p : 1.0 / p;
}

/* sym = 0: nk_triang (nk_moments.f90:105); sym = 1: mk_triang (mk_moments.f90:96),
   the same cell integral returned as a + transpose(a) */
static void nkmk_triang(const orc_basis *b, int k, int iv, double *rkd_iv, int sym)
{
    int ks = b->ks;
    int ik = ks * (ks + 1) / 2;
    int left = iv + ks - 1;
    double xbase = b->t[left];
    double gx[MAXKS], gw[MAXKS], bt[MAXKS * MAXKS], db[MAXKS], g2[MAXKS];
    double *INT = (double *)malloc(sizeof(double) * ks * ks * ks);
    for (int m = 0; m < ks; m++) {
        double span = GR(b, iv, m) - xbase;
        for (int i = 0; i < ks; i++) gx[i] = span * b->gx[i] + xbase;
        for (int i = 0; i < ks; i++) {
            orc_bsplvd(b->t, ks, gx[i], left, 1, db);
            for (int j = 0; j < ks; j++) bt[i + ks * j] = db[j];
        }
        for (int i = 0; i < ks; i++) gw[i] = span * b->gw[i] * ipow(gx[i], k);
        double c = GRW(b, iv, m) * ipow(GRM(b, iv, m), k + 3);
        for (int j = 0; j < ks; j++) {
            for (int i = 0; i < ks; i++) g2[i] = gw[i] * bt[i + ks * j];
            for (int jp = j; jp < ks; jp++) {
                double s = 0.0;
                for (int i = 0; i < ks; i++) s = s + g2[i] * bt[i + ks * jp];
                INT[j + ks * (jp + ks * m)] = s * c;
            }
        }
    }
    int ii = 0;
    for (int i = 0; i < ks; i++)
        for (int ip = i; ip < ks; ip++) {
            double g3[MAXKS];
            for (int m = 0; m < ks; m++) g3[m] = BSP(b, iv, m, i) * BSP(b, iv, m, ip);
            int jj = 0;
            for (int j = 0; j < ks; j++)
                for (int jp = j; jp < ks; jp++) {
                    double s = 0.0;
                    for (int m = 0; m < ks; m++) s = s + g3[m] * INT[j + ks * (jp + ks * m)];
                    rkd_iv[ii + ik * jj] = s;
                    jj++;
                }
            ii++;
        }
    if (sym) {
        double *a = (double *)malloc(sizeof(double) * ik * ik);
        memcpy(a, rkd_iv, sizeof(double) * ik * ik);
        for (int c = 0; c < ik; c++)
            for (int r = 0; r < ik; r++) rkd_iv[r + ik * c] = a[r + ik * c] + a[c + ik * r];
        free(a);
    }
    free(INT);
}

void orc_nk_triang(const orc_basis *b, int k, int iv, double *rkd_iv) { nkmk_triang(b, k, iv, rkd_iv, 0); }

static void nkmk_moments(const orc_basis *b, int k, double *rkd1, double *rkd2, double *rkd, int sym)
{
    int ks = b->ks, nv = b->nv, ml = b->ml, me = b->me;
    int ik = ks * (ks + 1) / 2;
    orc_moments(b, k, rkd1, 's', 'b');
    orc_moments(b, -(k + 3), rkd2, 's', 'b');
    size_t cell = (size_t)ik * ik;
    if (me == 0) {
        for (int iv = 0; iv < nv; iv++) nkmk_triang(b, k, iv, rkd + cell * iv, sym);
        return;
    }
    for (int iv = 1; iv <= ml + ks - 1 && iv <= nv; iv++) nkmk_triang(b, k, iv - 1, rkd + cell * (iv - 1), sym);
    double hp = b->h + 1.0;
    for (int iv = ml + ks; iv <= ml + me - ks + 2; iv++)
        for (size_t q = 0; q < cell; q++) rkd[q + cell * (iv - 1)] = rkd[q + cell * (iv - 2)] / hp;
    for (int iv = ml + me - ks + 3; iv <= nv; iv++)
        if (iv >= 1) nkmk_triang(b, k, iv - 1, rkd + cell * (iv - 1), sym);
}

void orc_nk_moments(const orc_basis *b, int k, double *rkd1, double *rkd2, double *rkd)
{
    nkmk_moments(b, k, rkd1, rkd2, rkd, 0);
}

/* mk_moments.f90:2: moments k and -(k+3) as for N^k, symmetrised diagonal cells */
void orc_mk_moments(const orc_basis *b, int k, double *rkd1, double *rkd2, double *rkd)
{
    nkmk_moments(b, k, rkd1, rkd2, rkd, 1);
}

/* mmk_cell.f90:2-83: mrk_cell's symmetric cell sums of the M^k moments, times fine */
void orc_mmk_cell(const orc_basis *b, int k, double fine, double *rkb, int ldp)
{
    int ks = b->ks, nv = b->nv, ns = b->ns;
    int ik = ks * (ks + 1) / 2;
    double *rkd1 = (double *)malloc(sizeof(double) * ik * nv);
    double *rkd2 = (double *)malloc(sizeof(double) * ik * nv);
    double *rkd = (double *)malloc(sizeof(double) * ik * ik * nv);
    orc_mk_moments(b, k, rkd1, rkd2, rkd);
    orc_mrk_cell_from(b, rkd1, rkd2, rkd, rkb, ldp);
    size_t tot = (size_t)ns * ns * ldp * ldp;
    for (size_t q = 0; q < tot; q++) rkb[q] = rkb[q] * fine;
    free(rkd1); free(rkd2); free(rkd);
}

/* rkb(i,j,ip,jp): i, ip the r1 (outer) splines, j, jp the r2 < r1 ones */
void orc_mnk_cell_from(const orc_basis *b, const double *rkd1, const double *rkd2, const double *rkd, double fine,
                       double *rkb, int ldp)
{
    int ks = b->ks, ns = b->ns, nv = b->nv;
    int ik = ks * (ks + 1) / 2;
    size_t nn = (size_t)ns * ns;
    memset(rkb, 0, sizeof(double) * nn * ldp * ldp);
    for (int iv = 0; iv < nv; iv++) {
        int ii = 0;
        for (int ih = 0; ih < ks; ih++) {
            int i = iv + ih;
            for (int ihp = ih; ihp < ks; ihp++) {
                int ip = ihp - ih;
                for (int jv = 0; jv <= iv; jv++) {
                    int jj = 0;
                    for (int jh = 0; jh < ks; jh++) {
                        int j = jv + jh;
                        for (int jhp = jh; jhp < ks; jhp++) {
                            int jp = jhp - jh;
                            double c = (jv < iv) ? rkd2[ii + (size_t)ik * iv] * rkd1[jj + (size_t)ik * jv]
                                                 : rkd[ii + (size_t)ik * (jj + (size_t)ik * iv)];
                            size_t o = i + (size_t)ns * j + nn * (ip + (size_t)ldp * jp);
                            rkb[o] = rkb[o] + c;
                            jj++;
                        }
                    }
                }
                ii++;
            }
        }
    }
    for (size_t q = 0; q < nn * ldp * ldp; q++) rkb[q] = rkb[q] * fine;
}

void orc_mnk_cell(const orc_basis *b, int k, double fine, double *rkb, int ldp)
{
    int ks = b->ks, nv = b->nv;
    int ik = ks * (ks + 1) / 2;
    double *rkd1 = (double *)malloc(sizeof(double) * ik * nv);
    double *rkd2 = (double *)malloc(sizeof(double) * ik * nv);
    double *rkd = (double *)malloc(sizeof(double) * ik * ik * nv);
    orc_nk_moments(b, k, rkd1, rkd2, rkd);
    orc_mnk_cell_from(b, rkd1, rkd2, rkd, fine, rkb, ldp);
    free(rkd1); free(rkd2); free(rkd);
}

/* nk.f90:2-47 with meth 'c': sum a(i,ip) b(j,jp) rkb(i,j,ip,jp), a = p_i1 p_i2, b = p_j1 p_j2 */
double orc_nk(int ns, int ks, const double *rkb, int ldp, const double *pi1, const double *pj1, const double *pi2,
              const double *pj2)
{
    double *a = (double *)malloc(sizeof(double) * ns * ks), *bb = (double *)malloc(sizeof(double) * ns * ks);
    size_t nn = (size_t)ns * ns;
    orc_density(ns, ks, a, pi1, pi2, 's');
    orc_density(ns, ks, bb, pj1, pj2, 's');
    double nk = 0.0;
    for (int ip = 1; ip <= ks; ip++)
        for (int i = 1; i <= ns - ip + 1; i++) {
            double nkj = 0.0;
            for (int jp = 1; jp <= ks; jp++)
                for (int j = 1; j <= ns - jp + 1; j++)
                    nkj = nkj + bb[(j - 1) + (size_t)ns * (jp - 1)] *
                                rkb[(i - 1) + (size_t)ns * (j - 1) + nn * ((ip - 1) + (size_t)ldp * (jp - 1))];
            nk = nk + a[(i - 1) + (size_t)ns * (ip - 1)] * nkj;
        }
    free(a); free(bb);
    return nk;
}

/* ------------------------------------------------------------------------ */
/* Breit-Pauli T^k: tk_moments.f90:2-216 (moments k and -(k+1) of 'n' pairs  */
/* with the derivative operator, tk_triang :101 -- inner integral of         */
/* B_j (dB_jp/dr - B_jp/r) r^k, outer bsq grm^(k+1), symmetrised; tk_pdiag   */
/* divides by (1+h)) and mtk_cell.f90:2-86 (all (ih, ihp) pairs,             */
/* ip = ihp - ih + ks, times fine/(2k+1)).  Tables (ns, ns, ldp, ldp), ldp   */
/* >= 2ks-1; moments jk = ks*ks.                                             */
/* ------------------------------------------------------------------------ */
void orc_tk_triang(const orc_basis *b, int k, int iv, double *rkd_iv)
{
    int ks = b->ks, jk = ks * ks;
    int left = iv + ks - 1;
    double xbase = b->t[left];
    double gx[MAXKS], gw[MAXKS], bt[MAXKS * MAXKS], bd[MAXKS * MAXKS], db[2 * MAXKS];
    double *INT = (double *)malloc(sizeof(double) * ks * ks * ks);
    for (int m = 0; m < ks; m++) {
        double span = GR(b, iv, m) - xbase;
        for (int i = 0; i < ks; i++) gx[i] = span * b->gx[i] + xbase;
        for (int i = 0; i < ks; i++) {
            orc_bsplvd(b->t, ks, gx[i], left, 2, db);
            for (int j = 0; j < ks; j++) {
                bt[i + ks * j] = db[j];
                bd[i + ks * j] = db[j + ks] - bt[i + ks * j] / gx[i];
            }
        }
        for (int i = 0; i < ks; i++) gw[i] = span * b->gw[i];
        for (int i = 0; i < ks; i++) gx[i] = ipow(gx[i], k) * gw[i];
        for (int j = 0; j < ks; j++) {
            for (int i = 0; i < ks; i++) gw[i] = gx[i] * bt[i + ks * j];
            for (int jp = 0; jp < ks; jp++) {
                double s = 0.0;
                for (int i = 0; i < ks; i++) s = s + gw[i] * bd[i + ks * jp];
                INT[j + ks * (jp + ks * m)] = s;
            }
        }
    }
    double g2[MAXKS], bq[MAXKS * MAXKS];
    for (int m = 0; m < ks; m++) g2[m] = GRW(b, iv, m) * ipow(GRM(b, iv, m), k + 1);
    for (int ip = 0; ip < ks; ip++)
        for (int m = 0; m < ks; m++) bq[m + ks * ip] = BSQ(b, iv, m, ip) * g2[m];
    double *a = (double *)malloc(sizeof(double) * jk * jk);
    int ii = 0;
    for (int i = 0; i < ks; i++)
        for (int ip = 0; ip < ks; ip++) {
            double g3[MAXKS];
            for (int m = 0; m < ks; m++) g3[m] = BSP(b, iv, m, i) * bq[m + ks * ip];
            int jj = 0;
            for (int j = 0; j < ks; j++)
                for (int jp = 0; jp < ks; jp++) {
                    double s = 0.0;
                    for (int m = 0; m < ks; m++) s = s + g3[m] * INT[j + ks * (jp + ks * m)];
                    a[ii + jk * jj] = s;
                    jj++;
                }
            ii++;
        }
    for (int c = 0; c < jk; c++)
        for (int r = 0; r < jk; r++) rkd_iv[r + jk * c] = a[r + jk * c] + a[c + jk * r];
    free(a);
    free(INT);
}

void orc_tk_moments(const orc_basis *b, int k, double *rkd1, double *rkd2, double *rkd)
{
    int ks = b->ks, nv = b->nv, ml = b->ml, me = b->me;
    int jk = ks * ks;
    orc_moments(b, k, rkd1, 'n', 'd');
    orc_moments(b, -(k + 1), rkd2, 'n', 'd');
    size_t cell = (size_t)jk * jk;
    if (me == 0) {
        for (int iv = 0; iv < nv; iv++) orc_tk_triang(b, k, iv, rkd + cell * iv);
        return;
    }
    for (int iv = 1; iv <= ml + ks - 1 && iv <= nv; iv++) orc_tk_triang(b, k, iv - 1, rkd + cell * (iv - 1));
    double hp = b->h + 1.0;
    for (int iv = ml + ks; iv <= ml + me - ks + 2; iv++)
        for (size_t q = 0; q < cell; q++) rkd[q + cell * (iv - 1)] = rkd[q + cell * (iv - 2)] / hp;
    for (int iv = ml + me - ks + 3; iv <= nv; iv++)
        if (iv >= 1) orc_tk_triang(b, k, iv - 1, rkd + cell * (iv - 1));
}

void orc_mtk_cell_from(const orc_basis *b, int k, const double *rkd1, const double *rkd2, const double *rkd,
                       double fine, double *rkb, int ldp)
{
    int ks = b->ks, ns = b->ns, nv = b->nv, jk = ks * ks;
    size_t nn = (size_t)ns * ns;
    memset(rkb, 0, sizeof(double) * nn * ldp * ldp);
    for (int jv = 0; jv < nv; jv++) {
        int jj = 0;
        for (int jh = 0; jh < ks; jh++) {
            int j = jv + jh;
            for (int jhp = 0; jhp < ks; jhp++) {
                int jp = jhp - jh + ks - 1;
                for (int iv = 0; iv < nv; iv++) {
                    int ii = 0;
                    for (int ih = 0; ih < ks; ih++) {
                        int i = iv + ih;
                        for (int ihp = 0; ihp < ks; ihp++) {
                            int ip = ihp - ih + ks - 1;
                            double c;
                            if (iv < jv) c = rkd1[ii + (size_t)jk * iv] * rkd2[jj + (size_t)jk * jv];
                            else if (iv > jv) c = rkd1[jj + (size_t)jk * jv] * rkd2[ii + (size_t)jk * iv];
                            else c = rkd[ii + (size_t)jk * (jj + (size_t)jk * iv)];
                            size_t o = i + (size_t)ns * j + nn * (ip + (size_t)ldp * jp);
                            rkb[o] = rkb[o] + c;
                            ii++;
                        }
                    }
                }
                jj++;
            }
        }
    }
    double c = fine / (k + k + 1);
    for (size_t q = 0; q < nn * ldp * ldp; q++) rkb[q] = rkb[q] * c;
}

void orc_mtk_cell(const orc_basis *b, int k, double fine, double *rkb, int ldp)
{
    int ks = b->ks, nv = b->nv, jk = ks * ks;
    double *rkd1 = (double *)malloc(sizeof(double) * jk * nv);
    double *rkd2 = (double *)malloc(sizeof(double) * jk * nv);
    double *rkd = (double *)malloc(sizeof(double) * jk * jk * nv);
    orc_tk_moments(b, k, rkd1, rkd2, rkd);
    orc_mtk_cell_from(b, k, rkd1, rkd2, rkd, fine, rkb, ldp);
    free(rkd1); free(rkd2); free(rkd);
}

/* tk.f90:2-58 (meth 'c'): sum b(j,jp) a(i,ip) rkb(i,j,ip,jp), a, b 'n' densities (ns, 2ks-1) */
double orc_tk(int ns, int ks, const double *rkb, int ldp, const double *pi1, const double *pj1, const double *pi2,
              const double *pj2)
{
    int kk = ks + ks - 1;
    double *a = (double *)malloc(sizeof(double) * ns * kk), *bb = (double *)malloc(sizeof(double) * ns * kk);
    size_t nn = (size_t)ns * ns;
    orc_density(ns, ks, a, pi1, pi2, 'n');
    orc_density(ns, ks, bb, pj1, pj2, 'n');
    double tk = 0.0;
    for (int jp = 1; jp <= kk; jp++) {
        int jmin = 1 + ks - jp > 1 ? 1 + ks - jp : 1, jmax = ns + ks - jp < ns ? ns + ks - jp : ns;
        for (int j = jmin; j <= jmax; j++) {
            double tki = 0.0;
            for (int ip = 1; ip <= kk; ip++) {
                int imin = 1 + ks - ip > 1 ? 1 + ks - ip : 1, imax = ns + ks - ip < ns ? ns + ks - ip : ns;
                for (int i = imin; i <= imax; i++)
                    tki = tki + a[(i - 1) + (size_t)ns * (ip - 1)] *
                                rkb[(i - 1) + (size_t)ns * (j - 1) + nn * ((ip - 1) + (size_t)ldp * (jp - 1))];
            }
            tk = tk + bb[(j - 1) + (size_t)ns * (jp - 1)] * tki;
        }
    }
    free(a); free(bb);
    return tk;
}

/* ------------------------------------------------------------------------ */
/* Breit-Pauli V^k: vk_moments.f90:2-218 -- rkd1 = moments(k+1,'s','b'),     */
/* rkd2 = moments(-(k+2),'s','b'), rkd3 = moments(k,'n','d'), rkd4 =         */
/* moments(-(k+3),'n','d'); diagonal cells rkd(ii in ks*ks, jj in ik) from   */
/* two inner integrals (vk_triang :131); vk_pdiag divides by (1+h) -- and    */
/* mvk_cell.f90:2-83 (jj over ik pairs with jp = jhp - jh + 1, ii over all   */
/* ks*ks pairs with ip = ihp - ih + ks; times fine).                         */
/* ------------------------------------------------------------------------ */
/* mode 0: vk_triang (vk_moments.f90:131); mode 1: wk_triang (wk_moments.f90:116) --
   inner operator 2 dB/dr + k B/r instead of dB/dr - B/r, and the outer operator of the
   second part 2 dB/dr - (k+3) B/r (bspd, grm) instead of bsq */
static void vw_triang(const orc_basis *b, int k, int iv, double *rkd_iv, int mode)
{
    int ks = b->ks, jk = ks * ks;
    const int jall = (mode == 2);       /* qk_triang: (j, jp) over all ks*ks pairs */
    int left = iv + ks - 1;
    double xbase = b->t[left];
    double gx[MAXKS], gw[MAXKS], bt[MAXKS * MAXKS], bd[MAXKS * MAXKS], db[2 * MAXKS], bi[MAXKS];
    double *I1 = (double *)malloc(sizeof(double) * ks * ks * ks);
    double *I2 = (double *)malloc(sizeof(double) * ks * ks * ks);
    for (int m = 0; m < ks; m++) {
        double span = GR(b, iv, m) - xbase;
        for (int i = 0; i < ks; i++) gx[i] = span * b->gx[i] + xbase;
        for (int i = 0; i < ks; i++) {
            orc_bsplvd(b->t, ks, gx[i], left, 2, db);
            for (int j = 0; j < ks; j++) {
                bt[i + ks * j] = db[j];
                bd[i + ks * j] = mode ? 2 * db[j + ks] + k * bt[i + ks * j] / gx[i]
                                      : db[j + ks] - bt[i + ks * j] / gx[i];
            }
        }
        for (int i = 0; i < ks; i++) gw[i] = span * b->gw[i] * ipow(gx[i], k);
        double c = ipow(GRM(b, iv, m), k + 2) * GRW(b, iv, m);
        for (int i = 0; i < ks; i++) {
            for (int q = 0; q < ks; q++) bi[q] = gw[q] * bt[q + ks * i];
            for (int ip = 0; ip < ks; ip++) {
                double s = 0.0;
                for (int q = 0; q < ks; q++) s = s + bi[q] * bd[q + ks * ip];
                I1[i + ks * (ip + ks * m)] = s * c;
            }
        }
        for (int q = 0; q < ks; q++) gw[q] = gw[q] * gx[q];
        c = ipow(GRM(b, iv, m), k + 3) * GRW(b, iv, m);
        for (int j = 0; j < ks; j++) {
            for (int q = 0; q < ks; q++) bi[q] = gw[q] * bt[q + ks * j];
            for (int jp = 0; jp < ks; jp++) {
                double s = 0.0;
                for (int q = 0; q < ks; q++) s = s + bi[q] * bt[q + ks * jp];
                I2[j + ks * (jp + ks * m)] = s * c;
            }
        }
    }
    int jj = 0;
    for (int j = 0; j < ks; j++)
        for (int jp = jall ? 0 : j; jp < ks; jp++) {
            double g3[MAXKS];
            for (int m = 0; m < ks; m++) g3[m] = BSP(b, iv, m, j) * BSP(b, iv, m, jp);
            int ii = 0;
            for (int i = 0; i < ks; i++)
                for (int ip = 0; ip < ks; ip++) {
                    double s = 0.0;
                    for (int m = 0; m < ks; m++) s = s + g3[m] * I1[i + ks * (ip + ks * m)];
                    rkd_iv[ii + jk * jj] = s;
                    ii++;
                }
            jj++;
        }
    int ii = 0;
    for (int i = 0; i < ks; i++)
        for (int ip = 0; ip < ks; ip++) {
            double g3[MAXKS];
            for (int m = 0; m < ks; m++) {
                double op = mode ? 2 * BSPD(b, iv, m, ip, 0) - (k + 3) * GRM(b, iv, m) * BSP(b, iv, m, ip)
                                 : BSQ(b, iv, m, ip);
                g3[m] = BSP(b, iv, m, i) * op;
            }
            jj = 0;
            for (int j = 0; j < ks; j++)
                for (int jp = jall ? 0 : j; jp < ks; jp++) {
                    double s = 0.0;
                    for (int m = 0; m < ks; m++) s = s + g3[m] * I2[j + ks * (jp + ks * m)];
                    rkd_iv[ii + jk * jj] = rkd_iv[ii + jk * jj] + s;
                    jj++;
                }
            ii++;
        }
    free(I1);
    free(I2);
}

void orc_vk_triang(const orc_basis *b, int k, int iv, double *rkd_iv) { vw_triang(b, k, iv, rkd_iv, 0); }

static void vw_moments(const orc_basis *b, int k, double *rkd1, double *rkd2, double *rkd3, double *rkd4,
                       double *rkd, int mode)
{
    int ks = b->ks, nv = b->nv, ml = b->ml, me = b->me;
    int jk = ks * ks, ik = ks * (ks + 1) / 2;
    if (!mode) {
        orc_moments(b, k + 1, rkd1, 's', 'b');
        orc_moments(b, -(k + 2), rkd2, 's', 'b');
        orc_moments(b, k, rkd3, 'n', 'd');
        orc_moments(b, -(k + 3), rkd4, 'n', 'd');
    } else {
        /* wk_moments.f90:44-52 (qk_moments.f90:44-52 with 'n' for rkd1, rkd2):
           rkd3 = 2 m(k,'n','d') + (k+2) m(k-1,'n','b'),
           rkd4 = 2 m(-(k+3),'n','d') - (k+1) m(-(k+4),'n','b') */
        const char sj = mode == 2 ? 'n' : 's';
        double *tmp = (double *)malloc(sizeof(double) * jk * nv);
        orc_moments(b, k, rkd3, 'n', 'd');
        orc_moments(b, k - 1, tmp, 'n', 'b');
        for (size_t q = 0; q < (size_t)jk * nv; q++) rkd3[q] = 2 * rkd3[q] + (k + 2) * tmp[q];
        orc_moments(b, -(k + 2), rkd2, sj, 'b');
        orc_moments(b, -(k + 3), rkd4, 'n', 'd');
        orc_moments(b, -(k + 4), tmp, 'n', 'b');
        for (size_t q = 0; q < (size_t)jk * nv; q++) rkd4[q] = 2 * rkd4[q] - (k + 1) * tmp[q];
        orc_moments(b, k + 1, rkd1, sj, 'b');
        free(tmp);
    }
    size_t cell = (size_t)jk * (mode == 2 ? jk : ik);
    if (me == 0) {
        for (int iv = 0; iv < nv; iv++) vw_triang(b, k, iv, rkd + cell * iv, mode);
        return;
    }
    for (int iv = 1; iv <= ml + ks - 1 && iv <= nv; iv++) vw_triang(b, k, iv - 1, rkd + cell * (iv - 1), mode);
    double hp = b->h + 1.0;
    for (int iv = ml + ks; iv <= ml + me - ks + 2; iv++)
        for (size_t q = 0; q < cell; q++) rkd[q + cell * (iv - 1)] = rkd[q + cell * (iv - 2)] / hp;
    for (int iv = ml + me - ks + 3; iv <= nv; iv++)
        if (iv >= 1) vw_triang(b, k, iv - 1, rkd + cell * (iv - 1), mode);
}

void orc_vk_moments(const orc_basis *b, int k, double *rkd1, double *rkd2, double *rkd3, double *rkd4, double *rkd)
{
    vw_moments(b, k, rkd1, rkd2, rkd3, rkd4, rkd, 0);
}

/* qk_moments.f90:2-239: rkd1, rkd2 (ks*ks, nv), rkd3, rkd4 (ks*ks, nv), rkd (ks*ks, ks*ks, nv) */
void orc_qk_moments(const orc_basis *b, int k, double *rkd1, double *rkd2, double *rkd3, double *rkd4, double *rkd)
{
    vw_moments(b, k, rkd1, rkd2, rkd3, rkd4, rkd, 2);
}

/* mqk_cell.f90:2-86: all (jh, jhp) and (ih, ihp) pairs, ip = ihp - ih + ks, jp = jhp - jh + ks;
   each term added to rkb(i,j,ip,jp) and subtracted from rkb(j,i,jp,ip) in loop order; times fine */
void orc_mqk_cell(const orc_basis *b, int k, double fine, double *rkb, int ldp)
{
    int ks = b->ks, ns = b->ns, nv = b->nv, jk = ks * ks;
    double *rkd1 = (double *)malloc(sizeof(double) * jk * nv), *rkd2 = (double *)malloc(sizeof(double) * jk * nv);
    double *rkd3 = (double *)malloc(sizeof(double) * jk * nv), *rkd4 = (double *)malloc(sizeof(double) * jk * nv);
    double *rkd = (double *)malloc(sizeof(double) * jk * jk * nv);
    orc_qk_moments(b, k, rkd1, rkd2, rkd3, rkd4, rkd);
    size_t nn = (size_t)ns * ns;
    memset(rkb, 0, sizeof(double) * nn * ldp * ldp);
    for (int jv = 0; jv < nv; jv++) {
        int jj = 0;
        for (int jh = 0; jh < ks; jh++) {
            int j = jv + jh;
            for (int jhp = 0; jhp < ks; jhp++) {
                int jp = jhp - jh + ks - 1;
                for (int iv = 0; iv < nv; iv++) {
                    int ii = 0;
                    for (int ih = 0; ih < ks; ih++) {
                        int i = iv + ih;
                        for (int ihp = 0; ihp < ks; ihp++) {
                            int ip = ihp - ih + ks - 1;
                            double c;
                            if (iv < jv) c = rkd3[ii + (size_t)jk * iv] * rkd2[jj + (size_t)jk * jv];
                            else if (iv > jv) c = rkd1[jj + (size_t)jk * jv] * rkd4[ii + (size_t)jk * iv];
                            else c = rkd[ii + (size_t)jk * (jj + (size_t)jk * iv)];
                            size_t o1 = i + (size_t)ns * j + nn * (ip + (size_t)ldp * jp);
                            size_t o2 = j + (size_t)ns * i + nn * (jp + (size_t)ldp * ip);
                            rkb[o1] = rkb[o1] + c;
                            rkb[o2] = rkb[o2] - c;
                            ii++;
                        }
                    }
                }
                jj++;
            }
        }
    }
    for (size_t q = 0; q < nn * ldp * ldp; q++) rkb[q] = rkb[q] * fine;
    free(rkd1); free(rkd2); free(rkd3); free(rkd4); free(rkd);
}

/* wk_moments.f90:2-241 */
void orc_wk_moments(const orc_basis *b, int k, double *rkd1, double *rkd2, double *rkd3, double *rkd4, double *rkd)
{
    vw_moments(b, k, rkd1, rkd2, rkd3, rkd4, rkd, 1);
}

/* rkb (ns, ns, ldp, ldp): ip up to 2ks-1 wide, jp up to ks; mode 0 mvk_cell, 1 mwk_cell (same sums) */
static void mvw_cell(const orc_basis *b, int k, double fine, double *rkb, int ldp, int mode)
{
    int ks = b->ks, ns = b->ns, nv = b->nv, jk = ks * ks, ik = ks * (ks + 1) / 2;
    double *rkd1 = (double *)malloc(sizeof(double) * ik * nv), *rkd2 = (double *)malloc(sizeof(double) * ik * nv);
    double *rkd3 = (double *)malloc(sizeof(double) * jk * nv), *rkd4 = (double *)malloc(sizeof(double) * jk * nv);
    double *rkd = (double *)malloc(sizeof(double) * jk * ik * nv);
    vw_moments(b, k, rkd1, rkd2, rkd3, rkd4, rkd, mode);
    size_t nn = (size_t)ns * ns;
    memset(rkb, 0, sizeof(double) * nn * ldp * ldp);
    for (int jv = 0; jv < nv; jv++) {
        int jj = 0;
        for (int jh = 0; jh < ks; jh++) {
            int j = jv + jh;
            for (int jhp = jh; jhp < ks; jhp++) {
                int jp = jhp - jh;
                for (int iv = 0; iv < nv; iv++) {
                    int ii = 0;
                    for (int ih = 0; ih < ks; ih++) {
                        int i = iv + ih;
                        for (int ihp = 0; ihp < ks; ihp++) {
                            int ip = ihp - ih + ks - 1;
                            double c;
                            if (iv < jv) c = rkd3[ii + (size_t)jk * iv] * rkd2[jj + (size_t)ik * jv];
                            else if (iv > jv) c = rkd1[jj + (size_t)ik * jv] * rkd4[ii + (size_t)jk * iv];
                            else c = rkd[ii + (size_t)jk * (jj + (size_t)ik * iv)];
                            size_t o = i + (size_t)ns * j + nn * (ip + (size_t)ldp * jp);
                            rkb[o] = rkb[o] + c;
                            ii++;
                        }
                    }
                }
                jj++;
            }
        }
    }
    for (size_t q = 0; q < nn * ldp * ldp; q++) rkb[q] = rkb[q] * fine;
    free(rkd1); free(rkd2); free(rkd3); free(rkd4); free(rkd);
}

void orc_mvk_cell(const orc_basis *b, int k, double fine, double *rkb, int ldp) { mvw_cell(b, k, fine, rkb, ldp, 0); }

/* mwk_cell.f90:2-83 */
void orc_mwk_cell(const orc_basis *b, int k, double fine, double *rkb, int ldp) { mvw_cell(b, k, fine, rkb, ldp, 1); }

/* vk.f90 (meth 'c'): a = 'n' density of (i1,i2), b = 's' density of (j1,j2) */
double orc_vk(int ns, int ks, const double *rkb, int ldp, const double *pi1, const double *pj1, const double *pi2,
              const double *pj2)
{
    int kk = ks + ks - 1;
    double *a = (double *)malloc(sizeof(double) * ns * kk), *bb = (double *)malloc(sizeof(double) * ns * ks);
    size_t nn = (size_t)ns * ns;
    orc_density(ns, ks, a, pi1, pi2, 'n');
    orc_density(ns, ks, bb, pj1, pj2, 's');
    double vk = 0.0;
    for (int jp = 1; jp <= ks; jp++)
        for (int j = 1; j <= ns - jp + 1; j++) {
            double vki = 0.0;
            for (int ip = 1; ip <= kk; ip++) {
                int imin = 1 + ks - ip > 1 ? 1 + ks - ip : 1, imax = ns + ks - ip < ns ? ns + ks - ip : ns;
                for (int i = imin; i <= imax; i++)
                    vki = vki + a[(i - 1) + (size_t)ns * (ip - 1)] *
                                rkb[(i - 1) + (size_t)ns * (j - 1) + nn * ((ip - 1) + (size_t)ldp * (jp - 1))];
            }
            vk = vk + bb[(j - 1) + (size_t)ns * (jp - 1)] * vki;
        }
    free(a); free(bb);
    return vk;
}
