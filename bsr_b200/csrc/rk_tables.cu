// B-spline basis tables and R^k cell tables on the GPU.
//
// Replaces, for the reference's B-spline library (src/libs/BS):
//   initvb  (define_spline.f90:67)  -> basis_points_kernel
//   mdb1/mdb2/mrm (define_spline.f90:184,214, mrm.f90:2) -> band_kernel
//   moments/moment (moments.f90:2,76) -> moments_kernel
//   rk_triang/rk_pdiag (rk_moments.f90:56,105) -> diag_cell_kernel
//   mrk_cell (mrk_cell.f90:2) -> rkb_expand_kernel
//
// This file is compiled with --fmad=false: every sum is accumulated in the
// reference's order with separately rounded multiplies and adds, so the tables
// equal the Fortran restatement's bit for bit.  All of it is one-shot or
// HBM-write bound (the rkb expansion), so giving up FMA costs nothing measurable.
#include "bsrg_internal.h"

namespace bsrg {

// de Boor's bsplvb/bsplvd (vbsplvd.f90:3,170) for one point.  left is the
// 0-based knot index with t[left] <= x <= t[left+1].  db[j + k*m] = m-th
// derivative of the j-th of the k B-splines nonzero on that interval.
struct BvbState {
    int j;
    double deltal[BSRG_MAXKS + 1], deltar[BSRG_MAXKS + 1];
};

__device__ static void bsplvb_dev(const double *t, int jhigh, int index, double x, int left,
                                           double *biatx, BvbState &st)
{
    if (index == 1) {
        st.j = 1;
        biatx[0] = 1.0;
        if (st.j >= jhigh) return;
    }
    for (;;) {
        int j = st.j, jp1 = j + 1;
        st.deltar[j - 1] = t[left + j] - x;
        st.deltal[j - 1] = x - t[left + 1 - j];
        double saved = 0.0;
        for (int i = 1; i <= j; i++) {
            double term = biatx[i - 1] / (st.deltar[i - 1] + st.deltal[jp1 - i - 1]);
            biatx[i - 1] = saved + st.deltar[i - 1] * term;
            saved = st.deltal[jp1 - i - 1] * term;
        }
        biatx[jp1 - 1] = saved;
        st.j = jp1;
        if (st.j >= jhigh) break;
    }
}

__device__ static void bsplvd_dev(const double *t, int k, double x, int left, int nderiv, double *db)
{
    BvbState st;
    int mhigh = nderiv < k ? nderiv : k;
    if (mhigh < 1) mhigh = 1;
    int kp1 = k + 1;
    bsplvb_dev(t, kp1 - mhigh, 1, x, left, db, st);
    if (mhigh == 1) return;
    int ideriv = mhigh;
    for (int m = 2; m <= mhigh; m++) {
        int jp1mid = 1;
        for (int j = ideriv; j <= k; j++) {
            db[(j - 1) + k * (ideriv - 1)] = db[jp1mid - 1];
            jp1mid++;
        }
        ideriv--;
        bsplvb_dev(t, kp1 - ideriv, 2, x, left, db, st);
    }
    double a[BSRG_MAXKS * BSRG_MAXKS];
#define A(i, j) a[((i) - 1) + k * ((j) - 1)]
    int jlow = 1;
    for (int i = 1; i <= k; i++) {
        for (int j = jlow; j <= k; j++) A(j, i) = 0.0;
        jlow = i;
        A(i, i) = 1.0;
    }
    for (int m = 2; m <= mhigh; m++) {
        int kp1mm = kp1 - m;
        double fk = (double)kp1mm;
        int il = left, i = k;
        for (int ld = 1; ld <= kp1mm; ld++) {
            double factor = fk / (t[il + kp1mm] - t[il]);
            for (int j = 1; j <= i; j++) A(i, j) = (A(i, j) - A(i - 1, j)) * factor;
            il--;
            i--;
        }
        for (int ii = 1; ii <= k; ii++) {
            double sum = 0.0;
            int jl = ii > m ? ii : m;
            for (int j = jl; j <= k; j++) sum = sum + A(j, ii) * db[(j - 1) + k * (m - 1)];
            db[(ii - 1) + k * (m - 1)] = sum;
        }
    }
#undef A
}

// values of the ks B-splines at x (nderiv = 1), no derivative work array
__device__ static void bspl_values(const double *t, int k, double x, int left, double *v)
{
    BvbState st;
    bsplvb_dev(t, k, 1, x, left, v, st);
}

// ---------------------------------------------------------------------------
// initvb: one thread per (interval, Gauss point); thread nv*ks does the last knot.
// ---------------------------------------------------------------------------
struct GaussRule { double x[BSRG_MAXKS], w[BSRG_MAXKS]; };

__global__ void basis_points_kernel(int ks, int ns, int nv, const double *__restrict__ t, GaussRule g,
                                    double *gr, double *grm, double *grw, double *bsp, double *bsq,
                                    double *bspd)
{
    int tid = blockIdx.x * blockDim.x + threadIdx.x;
    double db[BSRG_MAXKS * 3];
    size_t ld = (size_t)(nv + 1);
    if (tid < nv * ks) {
        int iv = tid % nv, m = tid / nv;
        double tl = t[iv + ks - 1], tr = t[iv + ks];
        double x = (tr - tl) * g.x[m] + tl;
        double xm = 1.0 / x;
        gr[iv + (size_t)nv * m] = x;
        grm[iv + (size_t)nv * m] = xm;
        grw[iv + (size_t)nv * m] = (tr - tl) * g.w[m];
        bsplvd_dev(t, ks, x, iv + ks - 1, 3, db);
        for (int ith = 0; ith < ks; ith++) {
            size_t o = iv + ld * (m + (size_t)ks * ith);
            double v = db[ith], d1 = db[ith + ks], d2 = db[ith + 2 * ks];
            bsp[o] = v;
            bspd[o] = d1;
            bspd[o + ld * ks * ks] = d2;
            bsq[o] = d1 - xm * v;
        }
    } else if (tid == nv * ks) {
        double x = t[ns];
        bsplvd_dev(t, ks, x, ns - 1, 3, db);
        for (int ith = 0; ith < ks; ith++) {
            size_t o = nv + ld * (0 + (size_t)ks * ith);
            double v = db[ith], d1 = db[ith + ks], d2 = db[ith + 2 * ks];
            bsp[o] = v;
            bspd[o] = d1;
            bspd[o + ld * ks * ks] = d2;
            bsq[o] = d1 - v / x;
        }
    }
}

// ---------------------------------------------------------------------------
// Band operator matrices in lower-column storage, one thread per (irow, jcol):
//   kind 0: <B_i|r^mm|B_j> (mrm.f90), kind 1: <B_i|B'_j> (mdb1), kind 2: <B_i|B''_j> (mdb2).
// The reference accumulates over ith = 1..ks (outer loop) for a fixed element.
// ---------------------------------------------------------------------------
__device__ static double rpow_dev(double g, int p)
{
    double r = g;
    for (int q = 1; q < p; q++) r = r * g;
    return r;
}

__global__ void band_kernel(int ks, int ns, int nv, int kind, int mm, const double *__restrict__ gr,
                            const double *__restrict__ grm, const double *__restrict__ grw,
                            const double *__restrict__ bsp, const double *__restrict__ bspd, double *out)
{
    int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= ns * ks) return;
    int irow = tid % ns, jcol = tid / ns;
    size_t ld = (size_t)(nv + 1);
    double acc = 0.0;
    for (int ith = 0; ith < ks; ith++) {
        int iv = irow - ith;
        int jth = jcol + ith - (ks - 1);
        if (iv < 0 || iv >= nv || jth < 0 || jth > ith) continue;
        double s = 0.0;
        for (int m = 0; m < ks; m++) {
            double w = grw[iv + (size_t)nv * m];
            double bi = bsp[iv + ld * (m + (size_t)ks * ith)];
            double wb = w * bi, v;
            if (kind == 0) {
                double bj = bsp[iv + ld * (m + (size_t)ks * jth)];
                if (mm == 0) v = wb * bj;
                else if (mm == -1) v = wb * grm[iv + (size_t)nv * m] * bj;
                else if (mm <= -2) v = wb * rpow_dev(grm[iv + (size_t)nv * m], -mm) * bj;
                else if (mm == 1) v = wb * gr[iv + (size_t)nv * m] * bj;
                else v = wb * rpow_dev(gr[iv + (size_t)nv * m], mm) * bj;
            } else {
                double dj = bspd[iv + ld * (m + (size_t)ks * (jth + (size_t)ks * (kind - 1)))];
                v = wb * dj;
            }
            s = s + v;
        }
        acc = acc + s;
    }
    if (kind == 2 && tid == 0) {
        // db2(1,1) holds <B_{ns-1}|B''_{ns}> over the last interval (define_spline.f90:238)
        int iv = nv - 1;
        double s = 0.0;
        for (int m = 0; m < ks; m++)
            s = s + grw[iv + (size_t)nv * m] * bsp[iv + ld * (m + (size_t)ks * (ks - 2))] *
                        bspd[iv + ld * (m + (size_t)ks * ((ks - 1) + (size_t)ks * 1))];
        acc = acc + s;
    }
    out[irow + (size_t)ns * jcol] = acc;
}

// ---------------------------------------------------------------------------
// moments (moments.f90:2,76), sym 's', dir 'b': rkm(ii, iv), one thread each.
// With me > 0 the geometric region repeats the reference's scaling chain
// rkm(:,iv) = rkm(:,iv-1)*hp starting from the last directly computed cell.
// ---------------------------------------------------------------------------
__device__ static double moment_one(int ks, int nv, int iv, int k, int i, int j, const double *gr,
                                    const double *grm, const double *grw, const double *bsp)
{
    size_t ld = (size_t)(nv + 1);
    double s = 0.0;
    for (int m = 0; m < ks; m++) {
        double gw = grw[iv + (size_t)nv * m];
        if (k > 0) gw = grw[iv + (size_t)nv * m] * rpow_dev(gr[iv + (size_t)nv * m], k);
        if (k < 0) gw = grw[iv + (size_t)nv * m] * rpow_dev(grm[iv + (size_t)nv * m], -k);
        double bj = bsp[iv + ld * (m + (size_t)ks * j)] * gw;
        s = s + bsp[iv + ld * (m + (size_t)ks * i)] * bj;
    }
    return s;
}

__global__ void moments_kernel(int ks, int nv, int ml, int me, double hp, int k, const double *gr,
                               const double *grm, const double *grw, const double *bsp, double *rkm)
{
    int ik = ks * (ks + 1) / 2;
    int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= ik * nv) return;
    int ii = tid % ik, iv = tid / ik;
    // unpack ii -> (i, j), i <= j
    int i = 0, rem = ii;
    while (rem >= ks - i) { rem -= ks - i; i++; }
    int j = i + rem;
    int iv1 = iv + 1;                        // 1-based
    int s0 = ml + ks, s1 = ml + me - ks + 2;  // scaled range (1-based), empty when me == 0
    double v;
    if (me != 0 && iv1 >= s0 && iv1 <= s1) {
        v = moment_one(ks, nv, s0 - 2, k, i, j, gr, grm, grw, bsp);
        for (int q = s0; q <= iv1; q++) v = v * hp;
    } else {
        v = moment_one(ks, nv, iv, k, i, j, gr, grm, grw, bsp);
    }
    rkm[ii + (size_t)ik * iv] = v;
}

// ---------------------------------------------------------------------------
// rk_triang (rk_moments.f90:105): one CTA per diagonal cell.  With me > 0 the
// cells of the geometric region repeat rk_pdiag's chain rkd(iv) = rkd(iv-1)*(1+h).
// ---------------------------------------------------------------------------
__global__ void diag_cell_kernel(int ks, int nv, int ml, int me, double hscale, int k,
                                 const double *__restrict__ t, GaussRule g, const double *gr,
                                 const double *grm, const double *grw, const double *bsp, double *rkd)
{
    extern __shared__ double sm[];
    const int ik = ks * (ks + 1) / 2;
    double *bt = sm;                          // [m][i][j] : ks*ks*ks  B-spline values at inner points
    double *wx = bt + ks * ks * ks;           // [m][i]   : weights * x^k at inner points
    double *INT = wx + ks * ks;               // [m][jj]  : ks*ik
    double *a = INT + ks * ik;                // [jj][ii] : ik*ik  (column-major a(ii,jj))
    double *BI = a + ik * ik;                 // [ii][m]  : ik*ks  bsp(i)*bsp(ip)*grw*grm^(k+1)
    int iv_out = blockIdx.x;
    int iv1 = iv_out + 1;
    int s0 = ml + ks, s1 = ml + me - ks + 2;
    int nscale = 0, iv = iv_out;
    if (me != 0 && iv1 >= s0 && iv1 <= s1) { iv = s0 - 2; nscale = iv1 - s0 + 1; }
    int left = iv + ks - 1;
    double xbase = t[left];
    size_t ld = (size_t)(nv + 1);
    // inner points: for each outer Gauss point m, ks points on [t_left, gr(iv,m)]
    for (int q = threadIdx.x; q < ks * ks; q += blockDim.x) {
        int m = q / ks, i = q % ks;
        double span = gr[iv + (size_t)nv * m] - xbase;
        double x = span * g.x[i] + xbase;
        double v[BSRG_MAXKS];
        bspl_values(t, ks, x, left, v);
        for (int j = 0; j < ks; j++) bt[(m * ks + i) * ks + j] = v[j];
        double w = span * g.w[i];
        double xk;
        if (k > 1) xk = w * rpow_dev(x, k);
        else if (k == 1) xk = w * x;
        else xk = w;
        wx[m * ks + i] = xk;
    }
    __syncthreads();
    // INT(j,jp,m) = SUM_i (wx_i * bt(i,j)) * bt(i,jp)
    for (int q = threadIdx.x; q < ks * ik; q += blockDim.x) {
        int m = q / ik, jj = q % ik;
        int j = 0, rem = jj;
        while (rem >= ks - j) { rem -= ks - j; j++; }
        int jp = j + rem;
        double s = 0.0;
        for (int i = 0; i < ks; i++) {
            double tmp = wx[m * ks + i] * bt[(m * ks + i) * ks + j];
            s = s + tmp * bt[(m * ks + i) * ks + jp];
        }
        INT[m * ik + jj] = s;
    }
    __syncthreads();
    // bi(ii,m) = bsp(i)*bsp(ip)*grw*grm^(k+1), once per cell
    for (int q = threadIdx.x; q < ik * ks; q += blockDim.x) {
        int ii = q / ks, m = q % ks;
        int i = 0, rem = ii;
        while (rem >= ks - i) { rem -= ks - i; i++; }
        int ip = i + rem;
        double g2;
        if (k != 0) g2 = grw[iv + (size_t)nv * m] * rpow_dev(grm[iv + (size_t)nv * m], k + 1);
        else g2 = grw[iv + (size_t)nv * m] * grm[iv + (size_t)nv * m];
        BI[q] = bsp[iv + ld * (m + (size_t)ks * i)] * bsp[iv + ld * (m + (size_t)ks * ip)] * g2;
    }
    __syncthreads();
    // a(ii,jj) = SUM_m bi(ii,m) * INT(jj,m)
    for (int q = threadIdx.x; q < ik * ik; q += blockDim.x) {
        int ii = q % ik, jj = q / ik;
        const double *bi = BI + ii * ks;
        double s = 0.0;
        for (int m = 0; m < ks; m++) s = s + bi[m] * INT[m * ik + jj];
        a[ii + ik * jj] = s;
    }
    __syncthreads();
    double *out = rkd + (size_t)ik * ik * iv_out;
    for (int q = threadIdx.x; q < ik * ik; q += blockDim.x) {
        int r = q % ik, c = q / ik;
        double v = a[r + ik * c] + a[c + ik * r];
        for (int n = 0; n < nscale; n++) v = v * hscale;
        out[r + (size_t)ik * c] = v;
    }
}

// ---------------------------------------------------------------------------
// mrk_cell (mrk_cell.f90:2): rkb(i,j,ip,jp) = sum over cells, jv outer and iv
// inner in ascending order as the reference accumulates.  One thread per
// element; a CTA covers 32 rows i (threadIdx.x, the contiguous index) x 8
// columns j for one (ip, jp).  The interval moments the CTA needs,
//   u1/u2[ih][iv] = rkd1/rkd2(pair (ih, ih+ip), iv) and w1/w2 likewise for jp,
// are staged in shared memory once, so the inner loop is two shared loads and
// a multiply-add per cell; only the diagonal cells (iv == jv) read rkd from
// global memory.  Elements with ip or jp >= ks (ldp > ks) or past the last
// spline are written as zero.
// ---------------------------------------------------------------------------
constexpr int EXP_TI = 32, EXP_TJ = 8;

__global__ void __launch_bounds__(EXP_TI * EXP_TJ)
rkb_expand_kernel(int ks, int ns, int nv, int ldp, double fine, const double *__restrict__ rkd1,
                  const double *__restrict__ rkd2, const double *__restrict__ rkd, double *__restrict__ rkb)
{
    extern __shared__ double sm[];
    const int ip = blockIdx.z % ldp, jp = blockIdx.z / ldp;
    const int i0 = blockIdx.x * EXP_TI, j0 = blockIdx.y * EXP_TJ;
    const int i = i0 + threadIdx.x, j = j0 + threadIdx.y;
    const int ik = ks * (ks + 1) / 2;
    const int LI = EXP_TI + ks - 1, LJ = EXP_TJ + ks - 1;     // interval windows
    const int ivb = i0 - (ks - 1), jvb = j0 - (ks - 1);       // first interval of each window
    double *u1 = sm, *u2 = u1 + ks * LI, *w1 = u2 + ks * LI, *w2 = w1 + ks * LJ;
    const bool active = ip < ks && jp < ks;
    if (active) {
        const int tid = threadIdx.y * EXP_TI + threadIdx.x, nt = EXP_TI * EXP_TJ;
        for (int q = tid; q < ks * LI; q += nt) {
            int ih = q / LI, iv = ivb + q % LI;
            double a = 0.0, b = 0.0;
            if (ih + ip < ks && iv >= 0 && iv < nv) {
                int ii = ih * ks - ih * (ih - 1) / 2 + ip;
                a = rkd1[ii + (size_t)ik * iv];
                b = rkd2[ii + (size_t)ik * iv];
            }
            u1[q] = a;
            u2[q] = b;
        }
        for (int q = tid; q < ks * LJ; q += nt) {
            int jh = q / LJ, jv = jvb + q % LJ;
            double a = 0.0, b = 0.0;
            if (jh + jp < ks && jv >= 0 && jv < nv) {
                int jj = jh * ks - jh * (jh - 1) / 2 + jp;
                a = rkd1[jj + (size_t)ik * jv];
                b = rkd2[jj + (size_t)ik * jv];
            }
            w1[q] = a;
            w2[q] = b;
        }
    }
    __syncthreads();
    if (i >= ns || j >= ns) return;
    double acc = 0.0;
    if (active && i + ip < ns && j + jp < ns) {
        int iv_lo = i + ip - (ks - 1); if (iv_lo < 0) iv_lo = 0;
        int iv_hi = i < nv - 1 ? i : nv - 1;
        int jv_lo = j + jp - (ks - 1); if (jv_lo < 0) jv_lo = 0;
        int jv_hi = j < nv - 1 ? j : nv - 1;
        for (int jv = jv_lo; jv <= jv_hi; jv++) {
            const int jh = j - jv, jl = jh * LJ + (jv - jvb);
            const double r2j = w2[jl], r1j = w1[jl];
            for (int iv = iv_lo; iv <= iv_hi; iv++) {
                const int ih = i - iv, il = ih * LI + (iv - ivb);
                double c;
                if (iv < jv) c = u1[il] * r2j;
                else if (iv > jv) c = r1j * u2[il];
                else {
                    int ii = ih * ks - ih * (ih - 1) / 2 + ip;
                    int jj = jh * ks - jh * (jh - 1) / 2 + jp;
                    c = rkd[ii + (size_t)ik * (jj + (size_t)ik * iv)];
                }
                acc = acc + c;
            }
        }
    }
    // fine = 1 for R^k (exact), spline_atomic's fine for M^k (mmk_cell.f90:79)
    rkb[i + (size_t)ns * (j + (size_t)ns * (ip + (size_t)ldp * jp))] = acc * fine;
}


// ---------------------------------------------------------------------------
// Breit-Pauli N^k tables.  nk_triang (nk_moments.f90:105): the diagonal cell of
// r2 < r1 only (inner weight r2^k, k >= -1; outer r1^-(k+3) folded into the
// inner integral), not symmetrised; nk_pdiag's scaling law divides by (1+h).
// ---------------------------------------------------------------------------
__device__ static double ipow_dev(double x, int k)
{
    if (k == 0) return 1.0;
    double p = x;
    const int a = k > 0 ? k : -k;
    for (int q = 1; q < a; q++) p = p * x;
    return k > 0 ? p : 1.0 / p;
}

__global__ void nk_diag_cell_kernel(int ks, int nv, int ml, int me, double hscale, int k, int sym,
                                    const double *__restrict__ t, GaussRule g, const double *gr,
                                    const double *grm, const double *grw, const double *bsp, double *rkd)
{
    extern __shared__ double sm[];
    const int ik = ks * (ks + 1) / 2;
    double *bt = sm;                          // [m][i][j] : B-spline values at the inner points
    double *wx = bt + ks * ks * ks;           // [m][i]   : inner weights * x^k
    double *INT = wx + ks * ks;               // [m][jj]
    double *a = INT + ks * ik;                // [jj][ii] (sym only): a(ii,jj) before a + a^T
    int iv_out = blockIdx.x;
    int iv1 = iv_out + 1;
    int s0 = ml + ks, s1 = ml + me - ks + 2;
    int nscale = 0, iv = iv_out;
    if (me != 0 && iv1 >= s0 && iv1 <= s1) { iv = s0 - 2; nscale = iv1 - s0 + 1; }
    int left = iv + ks - 1;
    double xbase = t[left];
    size_t ld = (size_t)(nv + 1);
    for (int q = threadIdx.x; q < ks * ks; q += blockDim.x) {
        int m = q / ks, i = q % ks;
        double span = gr[iv + (size_t)nv * m] - xbase;
        double x = span * g.x[i] + xbase;
        double v[BSRG_MAXKS];
        bspl_values(t, ks, x, left, v);
        for (int j = 0; j < ks; j++) bt[(m * ks + i) * ks + j] = v[j];
        wx[m * ks + i] = span * g.w[i] * ipow_dev(x, k);
    }
    __syncthreads();
    // INT(j,jp,m) = (SUM_i (wx_i bt(i,j)) bt(i,jp)) * grw(m) grm(m)^(k+3)
    for (int q = threadIdx.x; q < ks * ik; q += blockDim.x) {
        int m = q / ik, jj = q % ik;
        int j = 0, rem = jj;
        while (rem >= ks - j) { rem -= ks - j; j++; }
        int jp = j + rem;
        double s = 0.0;
        for (int i = 0; i < ks; i++) {
            double tmp = wx[m * ks + i] * bt[(m * ks + i) * ks + j];
            s = s + tmp * bt[(m * ks + i) * ks + jp];
        }
        const double c = grw[iv + (size_t)nv * m] * ipow_dev(grm[iv + (size_t)nv * m], k + 3);
        INT[m * ik + jj] = s * c;
    }
    __syncthreads();
    double *out = rkd + (size_t)ik * ik * iv_out;
    for (int q = threadIdx.x; q < ik * ik; q += blockDim.x) {
        int ii = q % ik, jj = q / ik;
        int i = 0, rem = ii;
        while (rem >= ks - i) { rem -= ks - i; i++; }
        int ip = i + rem;
        double s = 0.0;
        for (int m = 0; m < ks; m++) {
            double g3 = bsp[iv + ld * (m + (size_t)ks * i)] * bsp[iv + ld * (m + (size_t)ks * ip)];
            s = s + g3 * INT[m * ik + jj];
        }
        if (sym) {
            a[ii + ik * jj] = s;
        } else {
            for (int n = 0; n < nscale; n++) s = s / hscale;
            out[ii + (size_t)ik * jj] = s;
        }
    }
    if (!sym) return;
    // mk_triang (mk_moments.f90:96): the cell returned as a + transpose(a)
    __syncthreads();
    for (int q = threadIdx.x; q < ik * ik; q += blockDim.x) {
        int r = q % ik, c = q / ik;
        double v = a[r + ik * c] + a[c + ik * r];
        for (int n = 0; n < nscale; n++) v = v / hscale;
        out[r + (size_t)ik * c] = v;
    }
}

// mnk_cell (mnk_cell.f90:2): rkb(i,j,ip,jp) = fine * sum over cells iv (outer,
// r1) and jv <= iv (r2), in the reference's order; off-diagonal cells
// factorise as rkd2(ii,iv) rkd1(jj,jv).  Staging as in rkb_expand_kernel.
__global__ void __launch_bounds__(EXP_TI * EXP_TJ)
nkb_expand_kernel(int ks, int ns, int nv, int ldp, double fine, const double *__restrict__ rkd1,
                  const double *__restrict__ rkd2, const double *__restrict__ rkd, double *__restrict__ rkb)
{
    extern __shared__ double sm[];
    const int ip = blockIdx.z % ldp, jp = blockIdx.z / ldp;
    const int i0 = blockIdx.x * EXP_TI, j0 = blockIdx.y * EXP_TJ;
    const int i = i0 + threadIdx.x, j = j0 + threadIdx.y;
    const int ik = ks * (ks + 1) / 2;
    const int LI = EXP_TI + ks - 1, LJ = EXP_TJ + ks - 1;
    const int ivb = i0 - (ks - 1), jvb = j0 - (ks - 1);
    double *u2 = sm, *w1 = u2 + ks * LI;      // rkd2 on the r1 side, rkd1 on the r2 side
    const bool active = ip < ks && jp < ks;
    if (active) {
        const int tid = threadIdx.y * EXP_TI + threadIdx.x, nt = EXP_TI * EXP_TJ;
        for (int q = tid; q < ks * LI; q += nt) {
            int ih = q / LI, iv = ivb + q % LI;
            double b = 0.0;
            if (ih + ip < ks && iv >= 0 && iv < nv) b = rkd2[ih * ks - ih * (ih - 1) / 2 + ip + (size_t)ik * iv];
            u2[q] = b;
        }
        for (int q = tid; q < ks * LJ; q += nt) {
            int jh = q / LJ, jv = jvb + q % LJ;
            double a = 0.0;
            if (jh + jp < ks && jv >= 0 && jv < nv) a = rkd1[jh * ks - jh * (jh - 1) / 2 + jp + (size_t)ik * jv];
            w1[q] = a;
        }
    }
    __syncthreads();
    if (i >= ns || j >= ns) return;
    double acc = 0.0;
    if (active && i + ip < ns && j + jp < ns) {
        int iv_lo = i + ip - (ks - 1); if (iv_lo < 0) iv_lo = 0;
        int iv_hi = i < nv - 1 ? i : nv - 1;
        int jv_lo = j + jp - (ks - 1); if (jv_lo < 0) jv_lo = 0;
        int jv_hi = j < nv - 1 ? j : nv - 1;
        for (int iv = iv_lo; iv <= iv_hi; iv++) {
            const int ih = i - iv, il = ih * LI + (iv - ivb);
            const double r2i = u2[il];
            const int jmax = jv_hi < iv ? jv_hi : iv;
            for (int jv = jv_lo; jv <= jmax; jv++) {
                const int jh = j - jv;
                double c;
                if (jv < iv) c = r2i * w1[jh * LJ + (jv - jvb)];
                else {
                    int ii = ih * ks - ih * (ih - 1) / 2 + ip;
                    int jj = jh * ks - jh * (jh - 1) / 2 + jp;
                    c = rkd[ii + (size_t)ik * (jj + (size_t)ik * iv)];
                }
                acc = acc + c;
            }
        }
    }
    rkb[i + (size_t)ns * (j + (size_t)ns * (ip + (size_t)ldp * jp))] = acc * fine;
}


// ---------------------------------------------------------------------------
// Breit-Pauli T^k (tk_moments.f90, mtk_cell.f90).  moments 'n','d': all ks*ks
// pairs ii = i*ks + j with the derivative operator bsq on the second spline.
// ---------------------------------------------------------------------------
__global__ void moments_nd_kernel(int ks, int nv, int ml, int me, double hp, int k, const double *gr,
                                  const double *grm, const double *grw, const double *bsp, const double *bsq,
                                  double *rkm, int dir_b)
{
    const int jk = ks * ks;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= jk * nv) return;
    const int ii = tid % jk, iv_out = tid / jk;
    const int i = ii / ks, j = ii % ks;
    const int iv1 = iv_out + 1;
    const int s0 = ml + ks, s1 = ml + me - ks + 2;
    const bool scaled = me != 0 && iv1 >= s0 && iv1 <= s1;
    const int iv = scaled ? s0 - 2 : iv_out;
    const size_t ld = (size_t)(nv + 1);
    double v = 0.0;
    for (int m = 0; m < ks; m++) {
        double gw = grw[iv + (size_t)nv * m];
        if (k > 0) gw = grw[iv + (size_t)nv * m] * rpow_dev(gr[iv + (size_t)nv * m], k);
        if (k < 0) gw = grw[iv + (size_t)nv * m] * rpow_dev(grm[iv + (size_t)nv * m], -k);
        const double bj = (dir_b ? bsp : bsq)[iv + ld * (m + (size_t)ks * j)] * gw;
        v = v + bsp[iv + ld * (m + (size_t)ks * i)] * bj;
    }
    if (scaled)
        for (int q = s0; q <= iv1; q++) v = v * hp;
    rkm[ii + (size_t)jk * iv_out] = v;
}

// wk_moments.f90:44-52: out = 2 out + c tmp (c = k+2) or 2 out - c tmp (c = k+1)
__global__ void moments_combine_kernel(int n, double c, int minus, double *out, const double *tmp)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    out[q] = minus ? 2 * out[q] - c * tmp[q] : 2 * out[q] + c * tmp[q];
}

// tk_triang (tk_moments.f90:101): inner integral of B_j (dB_jp/dr - B_jp/r) r^k
// up to each outer Gauss point, outer weights bsq grw grm^(k+1), a + a^T.
__global__ void tk_diag_cell_kernel(int ks, int nv, int ml, int me, double hscale, int k,
                                    const double *__restrict__ t, GaussRule g, const double *gr,
                                    const double *grm, const double *grw, const double *bsp,
                                    const double *bsq, double *rkd)
{
    extern __shared__ double sm[];
    const int jk = ks * ks;
    double *bt = sm;                          // [m][i][j] values
    double *bd = bt + ks * ks * ks;           // [m][i][j] derivative - value/x
    double *wx = bd + ks * ks * ks;           // [m][i]
    double *INT = wx + ks * ks;               // [m][j][jp]
    double *bq = INT + ks * ks * ks;          // [m][ip]
    double *a = bq + ks * ks;                 // a(ii,jj), column-major jk x jk
    const int iv_out = blockIdx.x, iv1 = iv_out + 1;
    const int s0 = ml + ks, s1 = ml + me - ks + 2;
    int nscale = 0, iv = iv_out;
    if (me != 0 && iv1 >= s0 && iv1 <= s1) { iv = s0 - 2; nscale = iv1 - s0 + 1; }
    const int left = iv + ks - 1;
    const double xbase = t[left];
    const size_t ld = (size_t)(nv + 1);
    for (int q = threadIdx.x; q < ks * ks; q += blockDim.x) {
        const int m = q / ks, i = q % ks;
        const double span = gr[iv + (size_t)nv * m] - xbase;
        const double x = span * g.x[i] + xbase;
        double db[2 * BSRG_MAXKS];
        bsplvd_dev(t, ks, x, left, 2, db);
        for (int j = 0; j < ks; j++) {
            bt[(m * ks + i) * ks + j] = db[j];
            bd[(m * ks + i) * ks + j] = db[j + ks] - db[j] / x;
        }
        wx[m * ks + i] = ipow_dev(x, k) * (span * g.w[i]);
    }
    for (int q = threadIdx.x; q < ks * ks; q += blockDim.x) {
        const int m = q / ks, ip = q % ks;
        const double g2 = grw[iv + (size_t)nv * m] * ipow_dev(grm[iv + (size_t)nv * m], k + 1);
        bq[m * ks + ip] = bsq[iv + ld * (m + (size_t)ks * ip)] * g2;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < ks * jk; q += blockDim.x) {
        const int m = q / jk, j = (q % jk) / ks, jp = q % ks;
        double s = 0.0;
        for (int i = 0; i < ks; i++) {
            const double tmp = wx[m * ks + i] * bt[(m * ks + i) * ks + j];
            s = s + tmp * bd[(m * ks + i) * ks + jp];
        }
        INT[(m * ks + j) * ks + jp] = s;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < jk * jk; q += blockDim.x) {
        const int ii = q % jk, jj = q / jk;
        const int i = ii / ks, ip = ii % ks, j = jj / ks, jp = jj % ks;
        double s = 0.0;
        for (int m = 0; m < ks; m++) {
            const double g3 = bsp[iv + ld * (m + (size_t)ks * i)] * bq[m * ks + ip];
            s = s + g3 * INT[(m * ks + j) * ks + jp];
        }
        a[ii + jk * jj] = s;
    }
    __syncthreads();
    double *out = rkd + (size_t)jk * jk * iv_out;
    for (int q = threadIdx.x; q < jk * jk; q += blockDim.x) {
        const int r = q % jk, c = q / jk;
        double v = a[r + jk * c] + a[c + jk * r];
        for (int n = 0; n < nscale; n++) v = v / hscale;
        out[r + (size_t)jk * c] = v;
    }
}

// mtk_cell (mtk_cell.f90:2): rkb(i,j,ip,jp), ip = ihp - ih + ks - 1 (0-based, up
// to 2ks-2), summed over cells jv outer, iv inner; times fine/(2k+1).
__global__ void __launch_bounds__(EXP_TI * EXP_TJ)
tkb_expand_kernel(int ks, int ns, int nv, int ldp, double cfine, const double *__restrict__ rkd1,
                  const double *__restrict__ rkd2, const double *__restrict__ rkd, double *__restrict__ rkb)
{
    extern __shared__ double sm[];
    const int ip = blockIdx.z % ldp, jp = blockIdx.z / ldp;
    const int i0 = blockIdx.x * EXP_TI, j0 = blockIdx.y * EXP_TJ;
    const int i = i0 + threadIdx.x, j = j0 + threadIdx.y;
    const int jk = ks * ks;
    const int LI = EXP_TI + ks - 1, LJ = EXP_TJ + ks - 1;
    const int ivb = i0 - (ks - 1), jvb = j0 - (ks - 1);
    double *u1 = sm, *u2 = u1 + ks * LI, *w1 = u2 + ks * LI, *w2 = w1 + ks * LJ;
    const bool active = ip < 2 * ks - 1 && jp < 2 * ks - 1;
    if (active) {
        const int tid = threadIdx.y * EXP_TI + threadIdx.x, nt = EXP_TI * EXP_TJ;
        for (int q = tid; q < ks * LI; q += nt) {
            const int ih = q / LI, iv = ivb + q % LI, ihp = ih + ip - (ks - 1);
            double a = 0.0, b = 0.0;
            if (ihp >= 0 && ihp < ks && iv >= 0 && iv < nv) {
                a = rkd1[ih * ks + ihp + (size_t)jk * iv];
                b = rkd2[ih * ks + ihp + (size_t)jk * iv];
            }
            u1[q] = a;
            u2[q] = b;
        }
        for (int q = tid; q < ks * LJ; q += nt) {
            const int jh = q / LJ, jv = jvb + q % LJ, jhp = jh + jp - (ks - 1);
            double a = 0.0, b = 0.0;
            if (jhp >= 0 && jhp < ks && jv >= 0 && jv < nv) {
                a = rkd1[jh * ks + jhp + (size_t)jk * jv];
                b = rkd2[jh * ks + jhp + (size_t)jk * jv];
            }
            w1[q] = a;
            w2[q] = b;
        }
    }
    __syncthreads();
    if (i >= ns || j >= ns) return;
    double acc = 0.0;
    if (active) {
        // ih = i - iv with 0 <= ih < ks and 0 <= ih + ip - (ks-1) < ks
        const int ihmin = (ks - 1 - ip) > 0 ? ks - 1 - ip : 0, ihmax = (2 * ks - 2 - ip) < ks - 1 ? 2 * ks - 2 - ip : ks - 1;
        const int jhmin = (ks - 1 - jp) > 0 ? ks - 1 - jp : 0, jhmax = (2 * ks - 2 - jp) < ks - 1 ? 2 * ks - 2 - jp : ks - 1;
        int iv_lo = i - ihmax; if (iv_lo < 0) iv_lo = 0;
        int iv_hi = i - ihmin; if (iv_hi > nv - 1) iv_hi = nv - 1;
        int jv_lo = j - jhmax; if (jv_lo < 0) jv_lo = 0;
        int jv_hi = j - jhmin; if (jv_hi > nv - 1) jv_hi = nv - 1;
        for (int jv = jv_lo; jv <= jv_hi; jv++) {
            const int jh = j - jv, jl = jh * LJ + (jv - jvb);
            const double r2j = w2[jl], r1j = w1[jl];
            for (int iv = iv_lo; iv <= iv_hi; iv++) {
                const int ih = i - iv, il = ih * LI + (iv - ivb);
                double c;
                if (iv < jv) c = u1[il] * r2j;
                else if (iv > jv) c = r1j * u2[il];
                else {
                    const int ii = ih * ks + ih + ip - (ks - 1), jj = jh * ks + jh + jp - (ks - 1);
                    c = rkd[ii + (size_t)jk * (jj + (size_t)jk * iv)];
                }
                acc = acc + c;
            }
        }
    }
    rkb[i + (size_t)ns * (j + (size_t)ns * (ip + (size_t)ldp * jp))] = acc * cfine;
}


// ---------------------------------------------------------------------------
// Breit-Pauli V^k (vk_moments.f90, mvk_cell.f90).  vk_triang (:131): two inner
// integrals, I1(i,ip) of B_i (dB_ip/dr - B_ip/r) r^k with outer grm^(k+2), and
// I2(j,jp) of B_j B_jp r^(k+1) with outer grm^(k+3); rkd(ii = (i,ip) all pairs,
// jj = (j <= jp)) = sum bsp_j bsp_jp I1 + sum bsp_i bsq_ip I2.
// ---------------------------------------------------------------------------
__global__ void vk_diag_cell_kernel(int ks, int nv, int ml, int me, double hscale, int k, int mode,
                                    const double *__restrict__ t, GaussRule g, const double *gr,
                                    const double *grm, const double *grw, const double *bsp,
                                    const double *bsq, const double *bspd, double *rkd)
{
    extern __shared__ double sm[];
    const int jk = ks * ks, ik = ks * (ks + 1) / 2;
    double *bt = sm;                          // [m][q][j] values
    double *bd = bt + ks * ks * ks;           // [m][q][j] derivative - value/x
    double *w1 = bd + ks * ks * ks;           // [m][q] span w x^k
    double *w2 = w1 + ks * ks;                // [m][q] span w x^(k+1)
    double *I1 = w2 + ks * ks;                // [m][i][ip]
    double *I2 = I1 + ks * ks * ks;           // [m][j][jp]
    const int iv_out = blockIdx.x, iv1 = iv_out + 1;
    const int s0 = ml + ks, s1 = ml + me - ks + 2;
    int nscale = 0, iv = iv_out;
    if (me != 0 && iv1 >= s0 && iv1 <= s1) { iv = s0 - 2; nscale = iv1 - s0 + 1; }
    const int left = iv + ks - 1;
    const double xbase = t[left];
    const size_t ld = (size_t)(nv + 1);
    for (int q = threadIdx.x; q < ks * ks; q += blockDim.x) {
        const int m = q / ks, i = q % ks;
        const double span = gr[iv + (size_t)nv * m] - xbase;
        const double x = span * g.x[i] + xbase;
        double db[2 * BSRG_MAXKS];
        bsplvd_dev(t, ks, x, left, 2, db);
        for (int j = 0; j < ks; j++) {
            bt[(m * ks + i) * ks + j] = db[j];
            // V^k: dB/dr - B/r; W^k (wk_triang, wk_moments.f90:167): 2 dB/dr + k B/r
            bd[(m * ks + i) * ks + j] = mode ? 2 * db[j + ks] + (double)k * db[j] / x : db[j + ks] - db[j] / x;
        }
        const double w = span * g.w[i] * ipow_dev(x, k);
        w1[m * ks + i] = w;
        w2[m * ks + i] = w * x;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < ks * jk; q += blockDim.x) {
        const int m = q / jk, a = (q % jk) / ks, b = q % ks;
        const double gm = grm[iv + (size_t)nv * m], gwm = grw[iv + (size_t)nv * m];
        double s = 0.0, u = 0.0;
        for (int i = 0; i < ks; i++) {
            const double x1 = w1[m * ks + i] * bt[(m * ks + i) * ks + a];
            s = s + x1 * bd[(m * ks + i) * ks + b];
            const double x2 = w2[m * ks + i] * bt[(m * ks + i) * ks + a];
            u = u + x2 * bt[(m * ks + i) * ks + b];
        }
        I1[(m * ks + a) * ks + b] = s * (ipow_dev(gm, k + 2) * gwm);
        I2[(m * ks + a) * ks + b] = u * (ipow_dev(gm, k + 3) * gwm);
    }
    __syncthreads();
    // V^k, W^k: jj over the ik pairs j <= jp; Q^k (mode 2, qk_triang): over all ks*ks pairs
    const int njj = mode == 2 ? jk : ik;
    double *out = rkd + (size_t)jk * njj * iv_out;
    for (int q = threadIdx.x; q < jk * njj; q += blockDim.x) {
        const int ii = q % jk, jj = q / jk;
        const int i = ii / ks, ip = ii % ks;
        int j, jp;
        if (mode == 2) {
            j = jj / ks;
            jp = jj % ks;
        } else {
            j = 0;
            int rem = jj;
            while (rem >= ks - j) { rem -= ks - j; j++; }
            jp = j + rem;
        }
        double s1 = 0.0, s2 = 0.0;
        for (int m = 0; m < ks; m++) {
            const double g3 = bsp[iv + ld * (m + (size_t)ks * j)] * bsp[iv + ld * (m + (size_t)ks * jp)];
            s1 = s1 + g3 * I1[(m * ks + i) * ks + ip];
        }
        for (int m = 0; m < ks; m++) {
            // V^k: bsq; W^k (wk_moments.f90:218): 2 dB/dr - (k+3) B/r from the basis tables
            const double op = mode ? 2 * bspd[iv + ld * (m + (size_t)ks * ip)] -
                                         (double)(k + 3) * grm[iv + (size_t)nv * m] * bsp[iv + ld * (m + (size_t)ks * ip)]
                                   : bsq[iv + ld * (m + (size_t)ks * ip)];
            const double g3 = bsp[iv + ld * (m + (size_t)ks * i)] * op;
            s2 = s2 + g3 * I2[(m * ks + j) * ks + jp];
        }
        double v = s1 + s2;
        for (int n = 0; n < nscale; n++) v = v / hscale;
        out[ii + (size_t)jk * jj] = v;
    }
}

// mvk_cell (mvk_cell.f90:2): rkb(i,j,ip,jp), ip = ihp - ih + ks - 1 (0-based, up
// to 2ks-2) over all (ih, ihp), jp = jhp - jh over jh <= jhp; jv outer, iv
// inner; off-diagonal cells rkd3 x rkd2 (iv < jv) or rkd1 x rkd4; times fine.
__global__ void __launch_bounds__(EXP_TI * EXP_TJ)
vkb_expand_kernel(int ks, int ns, int nv, int ldp, double fine, const double *__restrict__ rkd1,
                  const double *__restrict__ rkd2, const double *__restrict__ rkd3,
                  const double *__restrict__ rkd4, const double *__restrict__ rkd, double *__restrict__ rkb)
{
    extern __shared__ double sm[];
    const int ip = blockIdx.z % ldp, jp = blockIdx.z / ldp;
    const int i0 = blockIdx.x * EXP_TI, j0 = blockIdx.y * EXP_TJ;
    const int i = i0 + threadIdx.x, j = j0 + threadIdx.y;
    const int jk = ks * ks, ik = ks * (ks + 1) / 2;
    const int LI = EXP_TI + ks - 1, LJ = EXP_TJ + ks - 1;
    const int ivb = i0 - (ks - 1), jvb = j0 - (ks - 1);
    double *u3 = sm, *u4 = u3 + ks * LI, *w1 = u4 + ks * LI, *w2 = w1 + ks * LJ;
    const bool active = ip < 2 * ks - 1 && jp < ks;
    if (active) {
        const int tid = threadIdx.y * EXP_TI + threadIdx.x, nt = EXP_TI * EXP_TJ;
        for (int q = tid; q < ks * LI; q += nt) {
            const int ih = q / LI, iv = ivb + q % LI, ihp = ih + ip - (ks - 1);
            double a = 0.0, b = 0.0;
            if (ihp >= 0 && ihp < ks && iv >= 0 && iv < nv) {
                a = rkd3[ih * ks + ihp + (size_t)jk * iv];
                b = rkd4[ih * ks + ihp + (size_t)jk * iv];
            }
            u3[q] = a;
            u4[q] = b;
        }
        for (int q = tid; q < ks * LJ; q += nt) {
            const int jh = q / LJ, jv = jvb + q % LJ;
            double a = 0.0, b = 0.0;
            if (jh + jp < ks && jv >= 0 && jv < nv) {
                const int jj = jh * ks - jh * (jh - 1) / 2 + jp;
                a = rkd1[jj + (size_t)ik * jv];
                b = rkd2[jj + (size_t)ik * jv];
            }
            w1[q] = a;
            w2[q] = b;
        }
    }
    __syncthreads();
    if (i >= ns || j >= ns) return;
    double acc = 0.0;
    if (active && j + jp < ns) {
        const int ihmin = (ks - 1 - ip) > 0 ? ks - 1 - ip : 0, ihmax = (2 * ks - 2 - ip) < ks - 1 ? 2 * ks - 2 - ip : ks - 1;
        int iv_lo = i - ihmax; if (iv_lo < 0) iv_lo = 0;
        int iv_hi = i - ihmin; if (iv_hi > nv - 1) iv_hi = nv - 1;
        int jv_lo = j + jp - (ks - 1); if (jv_lo < 0) jv_lo = 0;
        int jv_hi = j < nv - 1 ? j : nv - 1;
        for (int jv = jv_lo; jv <= jv_hi; jv++) {
            const int jh = j - jv, jl = jh * LJ + (jv - jvb);
            const double r1j = w1[jl], r2j = w2[jl];
            for (int iv = iv_lo; iv <= iv_hi; iv++) {
                const int ih = i - iv, il = ih * LI + (iv - ivb);
                double c;
                if (iv < jv) c = u3[il] * r2j;
                else if (iv > jv) c = r1j * u4[il];
                else {
                    const int ii = ih * ks + ih + ip - (ks - 1);
                    const int jj = jh * ks - jh * (jh - 1) / 2 + jp;
                    c = rkd[ii + (size_t)jk * (jj + (size_t)ik * iv)];
                }
                acc = acc + c;
            }
        }
    }
    rkb[i + (size_t)ns * (j + (size_t)ns * (ip + (size_t)ldp * jp))] = acc * fine;
}

// mqk_cell (mqk_cell.f90:2): the reference adds every cell term c to rkb(i,j,ip,jp)
// and subtracts it from rkb(j,i,jp,ip) within one loop (jv, jh, jhp outer; iv, ih,
// ihp inner).  For one element and one jv, all its added terms share (jh, jhp) and
// all its subtracted terms share another (jh, jhp), so per jv one block precedes the
// other in the reference's order; a self-transposed element gets +c then -c in the
// same iteration.  One thread per element replays that order, then times fine.
__device__ __forceinline__ double qk_term(int ks, int jk, int jv, int jh, int jhp, int iv, int ih, int ihp,
                                          const double *rkd1, const double *rkd2, const double *rkd3,
                                          const double *rkd4, const double *rkd)
{
    const int ii = ih * ks + ihp, jj = jh * ks + jhp;
    if (iv < jv) return rkd3[ii + (size_t)jk * iv] * rkd2[jj + (size_t)jk * jv];
    if (iv > jv) return rkd1[jj + (size_t)jk * jv] * rkd4[ii + (size_t)jk * iv];
    return rkd[ii + (size_t)jk * (jj + (size_t)jk * iv)];
}

__global__ void qkb_expand_kernel(int ks, int ns, int nv, int ldp, double fine, const double *__restrict__ rkd1,
                                  const double *__restrict__ rkd2, const double *__restrict__ rkd3,
                                  const double *__restrict__ rkd4, const double *__restrict__ rkd,
                                  double *__restrict__ rkb)
{
    const size_t nn = (size_t)ns * ns;
    const size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (q >= nn * ldp * ldp) return;
    const int I = (int)(q % ns), J = (int)((q / ns) % ns);
    const int IP = (int)((q / nn) % ldp), JP = (int)(q / (nn * ldp));
    const int jk = ks * ks, H = ks - 1;
    double acc = 0.0;
    if (IP < 2 * ks - 1 && JP < 2 * ks - 1) {
        const bool self = (I == J && IP == JP);
        int jv_lo = (I < J ? I : J) - H; if (jv_lo < 0) jv_lo = 0;
        int jv_hi = I > J ? I : J; if (jv_hi > nv - 1) jv_hi = nv - 1;
        for (int jv = jv_lo; jv <= jv_hi; jv++) {
            // added terms: (i,j,ip,jp) = (I,J,IP,JP); subtracted: (i,j,ip,jp) = (J,I,JP,IP)
            const int jhA = J - jv, jhpA = JP - H + jhA;
            const int jhS = I - jv, jhpS = IP - H + jhS;
            const bool vA = jhA >= 0 && jhA < ks && jhpA >= 0 && jhpA < ks;
            const bool vS = jhS >= 0 && jhS < ks && jhpS >= 0 && jhpS < ks;
            if (self) {
                if (!vA) continue;
                for (int iv = (I - H > 0 ? I - H : 0); iv <= I && iv < nv; iv++) {
                    const int ih = I - iv, ihp = IP - H + ih;
                    if (ihp < 0 || ihp >= ks) continue;
                    const double c = qk_term(ks, jk, jv, jhA, jhpA, iv, ih, ihp, rkd1, rkd2, rkd3, rkd4, rkd);
                    acc = acc + c;
                    acc = acc - c;
                }
                continue;
            }
            const bool addFirst = (jhA < jhS) || (jhA == jhS && jhpA < jhpS);
            for (int pass = 0; pass < 2; pass++) {
                const bool add = (pass == 0) == addFirst;
                if (add ? !vA : !vS) continue;
                const int Ir = add ? I : J, IPr = add ? IP : JP;       // the iteration's i and ip
                const int jh = add ? jhA : jhS, jhp = add ? jhpA : jhpS;
                for (int iv = (Ir - H > 0 ? Ir - H : 0); iv <= Ir && iv < nv; iv++) {
                    const int ih = Ir - iv, ihp = IPr - H + ih;
                    if (ihp < 0 || ihp >= ks) continue;
                    const double c = qk_term(ks, jk, jv, jh, jhp, iv, ih, ihp, rkd1, rkd2, rkd3, rkd4, rkd);
                    acc = add ? acc + c : acc - c;
                }
            }
        }
    }
    rkb[q] = acc * fine;
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static GaussRule rule_of(const bsrg_basis *b)
{
    GaussRule g;
    for (int i = 0; i < BSRG_MAXKS; i++) { g.x[i] = i < b->ks ? b->gx[i] : 0.0; g.w[i] = i < b->ks ? b->gw[i] : 0.0; }
    return g;
}

int launch_basis_tables(bsrg_basis *b, cudaStream_t s)
{
    int n = b->nv * b->ks + 1;
    basis_points_kernel<<<(n + 127) / 128, 128, 0, s>>>(b->ks, b->ns, b->nv, b->t, rule_of(b), b->gr, b->grm,
                                                         b->grw, b->bsp, b->bsq, b->bspd);
    int nb = b->ns * b->ks, bl = (nb + 127) / 128;
    band_kernel<<<bl, 128, 0, s>>>(b->ks, b->ns, b->nv, 1, 0, b->gr, b->grm, b->grw, b->bsp, b->bspd, b->db1);
    band_kernel<<<bl, 128, 0, s>>>(b->ks, b->ns, b->nv, 2, 0, b->gr, b->grm, b->grw, b->bsp, b->bspd, b->db2);
    band_kernel<<<bl, 128, 0, s>>>(b->ks, b->ns, b->nv, 0, 0, b->gr, b->grm, b->grw, b->bsp, b->bspd, b->sb);
    band_kernel<<<bl, 128, 0, s>>>(b->ks, b->ns, b->nv, 0, 1, b->gr, b->grm, b->grw, b->bsp, b->bspd, b->r1);
    band_kernel<<<bl, 128, 0, s>>>(b->ks, b->ns, b->nv, 0, -1, b->gr, b->grm, b->grw, b->bsp, b->bspd, b->rm1);
    band_kernel<<<bl, 128, 0, s>>>(b->ks, b->ns, b->nv, 0, -2, b->gr, b->grm, b->grw, b->bsp, b->bspd, b->rm2);
    band_kernel<<<bl, 128, 0, s>>>(b->ks, b->ns, b->nv, 0, -3, b->gr, b->grm, b->grw, b->bsp, b->bspd, b->rm3);
    return cuda_fail(cudaGetLastError(), "basis tables");
}

int launch_mrm(const bsrg_basis *b, int mm, double *rm, cudaStream_t s)
{
    int nb = b->ns * b->ks;
    band_kernel<<<(nb + 127) / 128, 128, 0, s>>>(b->ks, b->ns, b->nv, 0, mm, b->gr, b->grm, b->grw, b->bsp,
                                                 b->bspd, rm);
    return cuda_fail(cudaGetLastError(), "mrm");
}

static double ipow_host(double q, int k)
{
    double hp = 1.0;
    if (k >= 0) { for (int i = 0; i < k; i++) hp *= q; }
    else { double p = 1.0; for (int i = 0; i < -k; i++) p *= q; hp = 1.0 / p; }
    return hp;
}

int launch_rk_moments(const bsrg_basis *b, int k, double *rkd1, double *rkd2, double *rkd, cudaStream_t s)
{
    int ks = b->ks, nv = b->nv, ik = ik_of(ks);
    double q = 1.0 + b->h;
    int n = ik * nv;
    if (rkd1)
        moments_kernel<<<(n + 127) / 128, 128, 0, s>>>(ks, nv, b->ml, b->me, ipow_host(q, k) * q, k, b->gr,
                                                       b->grm, b->grw, b->bsp, rkd1);
    if (rkd2)
        moments_kernel<<<(n + 127) / 128, 128, 0, s>>>(ks, nv, b->ml, b->me, ipow_host(q, -(k + 1)) * q,
                                                       -(k + 1), b->gr, b->grm, b->grw, b->bsp, rkd2);
    if (rkd) {
        size_t shm = sizeof(double) * ((size_t)ks * ks * ks + ks * ks + 2 * (size_t)ks * ik + (size_t)ik * ik);
        if (shm > 48 * 1024) {
            cudaError_t e = smem_attr(diag_cell_kernel, (int)shm);
            if (e != cudaSuccess) return cuda_fail(e, "diag_cell smem");
        }
        diag_cell_kernel<<<nv, 256, shm, s>>>(ks, nv, b->ml, b->me, b->h + 1.0, k, b->t, rule_of(b), b->gr,
                                             b->grm, b->grw, b->bsp, rkd);
    }
    return cuda_fail(cudaGetLastError(), "rk_moments");
}

int launch_mrk_cell_scaled(const bsrg_basis *b, const double *rkd1, const double *rkd2, const double *rkd,
                           double fine, double *rkb, int ldp, cudaStream_t s)
{
    dim3 blk(EXP_TI, EXP_TJ);
    dim3 grd((b->ns + EXP_TI - 1) / EXP_TI, (b->ns + EXP_TJ - 1) / EXP_TJ, ldp * ldp);
    size_t shm = sizeof(double) * 2 * (size_t)b->ks * ((EXP_TI + b->ks - 1) + (EXP_TJ + b->ks - 1));
    rkb_expand_kernel<<<grd, blk, shm, s>>>(b->ks, b->ns, b->nv, ldp, fine, rkd1, rkd2, rkd, rkb);
    return cuda_fail(cudaGetLastError(), "mrk_cell");
}

int launch_mrk_cell(const bsrg_basis *b, const double *rkd1, const double *rkd2, const double *rkd,
                    double *rkb, int ldp, cudaStream_t s)
{
    return launch_mrk_cell_scaled(b, rkd1, rkd2, rkd, 1.0, rkb, ldp, s);
}

// N^k (sym = 0) or M^k (sym = 1) moments: the same moments, M^k symmetrises the diagonal cells
int launch_nkmk_moments(const bsrg_basis *b, int k, int sym, double *rkd1, double *rkd2, double *rkd,
                        cudaStream_t s)
{
    int ks = b->ks, nv = b->nv, ik = ik_of(ks);
    double q = 1.0 + b->h;
    int n = ik * nv;
    if (rkd1)
        moments_kernel<<<(n + 127) / 128, 128, 0, s>>>(ks, nv, b->ml, b->me, ipow_host(q, k) * q, k, b->gr,
                                                       b->grm, b->grw, b->bsp, rkd1);
    if (rkd2)
        moments_kernel<<<(n + 127) / 128, 128, 0, s>>>(ks, nv, b->ml, b->me, ipow_host(q, -(k + 3)) * q,
                                                       -(k + 3), b->gr, b->grm, b->grw, b->bsp, rkd2);
    if (rkd) {
        size_t shm = sizeof(double) * ((size_t)ks * ks * ks + ks * ks + (size_t)ks * ik + (sym ? (size_t)ik * ik : 0));
        if (shm > 48 * 1024) {
            cudaError_t e = smem_attr(nk_diag_cell_kernel, (int)shm);
            if (e != cudaSuccess) return cuda_fail(e, "nk diag_cell smem");
        }
        nk_diag_cell_kernel<<<nv, 256, shm, s>>>(ks, nv, b->ml, b->me, b->h + 1.0, k, sym, b->t, rule_of(b), b->gr,
                                                b->grm, b->grw, b->bsp, rkd);
    }
    return cuda_fail(cudaGetLastError(), sym ? "mk_moments" : "nk_moments");
}

int launch_mnk_cell(const bsrg_basis *b, const double *rkd1, const double *rkd2, const double *rkd, double fine,
                    double *rkb, int ldp, cudaStream_t s)
{
    dim3 blk(EXP_TI, EXP_TJ);
    dim3 grd((b->ns + EXP_TI - 1) / EXP_TI, (b->ns + EXP_TJ - 1) / EXP_TJ, ldp * ldp);
    size_t shm = sizeof(double) * (size_t)b->ks * ((EXP_TI + b->ks - 1) + (EXP_TJ + b->ks - 1));
    nkb_expand_kernel<<<grd, blk, shm, s>>>(b->ks, b->ns, b->nv, ldp, fine, rkd1, rkd2, rkd, rkb);
    return cuda_fail(cudaGetLastError(), "mnk_cell");
}

int launch_tk_moments(const bsrg_basis *b, int k, double *rkd1, double *rkd2, double *rkd, cudaStream_t s)
{
    const int ks = b->ks, nv = b->nv, jk = ks * ks;
    const double q = 1.0 + b->h;
    const int n = jk * nv;
    // dir 'd': the scaling law of the moments carries no extra (1+h) (moments.f90)
    if (rkd1)
        moments_nd_kernel<<<(n + 127) / 128, 128, 0, s>>>(ks, nv, b->ml, b->me, ipow_host(q, k), k, b->gr, b->grm,
                                                          b->grw, b->bsp, b->bsq, rkd1, 0);
    if (rkd2)
        moments_nd_kernel<<<(n + 127) / 128, 128, 0, s>>>(ks, nv, b->ml, b->me, ipow_host(q, -(k + 1)), -(k + 1),
                                                          b->gr, b->grm, b->grw, b->bsp, b->bsq, rkd2, 0);
    if (rkd) {
        const size_t shm = sizeof(double) * (3 * (size_t)ks * ks * ks + 2 * (size_t)ks * ks + (size_t)jk * jk);
        int dev = 0, optin = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        if (shm > (size_t)optin) {
            set_error("tk_moments: a diagonal cell of ks=%d needs %zu bytes of shared memory (device limit %d)", ks,
                      shm, optin);
            return BSRG_ERR_ARG;
        }
        cudaError_t e = smem_attr(tk_diag_cell_kernel, (int)shm);
        if (e != cudaSuccess) return cuda_fail(e, "tk diag_cell smem");
        tk_diag_cell_kernel<<<nv, 256, shm, s>>>(ks, nv, b->ml, b->me, b->h + 1.0, k, b->t, rule_of(b), b->gr,
                                                b->grm, b->grw, b->bsp, b->bsq, rkd);
    }
    return cuda_fail(cudaGetLastError(), "tk_moments");
}

int launch_mtk_cell(const bsrg_basis *b, int k, const double *rkd1, const double *rkd2, const double *rkd,
                    double fine, double *rkb, int ldp, cudaStream_t s)
{
    dim3 blk(EXP_TI, EXP_TJ);
    dim3 grd((b->ns + EXP_TI - 1) / EXP_TI, (b->ns + EXP_TJ - 1) / EXP_TJ, ldp * ldp);
    const size_t shm = sizeof(double) * 2 * (size_t)b->ks * ((EXP_TI + b->ks - 1) + (EXP_TJ + b->ks - 1));
    const double cfine = fine / (k + k + 1);
    tkb_expand_kernel<<<grd, blk, shm, s>>>(b->ks, b->ns, b->nv, ldp, cfine, rkd1, rkd2, rkd, rkb);
    return cuda_fail(cudaGetLastError(), "mtk_cell");
}

// mode 0: V^k (vk_moments.f90); mode 1: W^k (wk_moments.f90), tmp (ks*ks*nv) needed for the combinations
int launch_vw_moments(const bsrg_basis *b, int k, int mode, double *rkd1, double *rkd2, double *rkd3, double *rkd4,
                      double *rkd, double *tmp, cudaStream_t s)
{
    const int ks = b->ks, nv = b->nv, jk = ks * ks, ik = ik_of(ks);
    const double q = 1.0 + b->h;
    if (mode == 2) {        // qk_moments.f90: rkd1, rkd2 over all ks*ks pairs ('n','b')
        const int gq = (jk * nv + 127) / 128;
        if (rkd1)
            moments_nd_kernel<<<gq, 128, 0, s>>>(ks, nv, b->ml, b->me, ipow_host(q, k + 1) * q, k + 1, b->gr, b->grm,
                                                 b->grw, b->bsp, b->bsq, rkd1, 1);
        if (rkd2)
            moments_nd_kernel<<<gq, 128, 0, s>>>(ks, nv, b->ml, b->me, ipow_host(q, -(k + 2)) * q, -(k + 2), b->gr,
                                                 b->grm, b->grw, b->bsp, b->bsq, rkd2, 1);
    } else {
        if (rkd1)
            moments_kernel<<<(ik * nv + 127) / 128, 128, 0, s>>>(ks, nv, b->ml, b->me, ipow_host(q, k + 1) * q, k + 1,
                                                                  b->gr, b->grm, b->grw, b->bsp, rkd1);
        if (rkd2)
            moments_kernel<<<(ik * nv + 127) / 128, 128, 0, s>>>(ks, nv, b->ml, b->me, ipow_host(q, -(k + 2)) * q,
                                                                  -(k + 2), b->gr, b->grm, b->grw, b->bsp, rkd2);
    }
    const int nj = jk * nv, gj = (nj + 127) / 128;
    if (rkd3) {
        moments_nd_kernel<<<gj, 128, 0, s>>>(ks, nv, b->ml, b->me, ipow_host(q, k), k, b->gr, b->grm, b->grw, b->bsp,
                                             b->bsq, rkd3, 0);
        if (mode) {
            moments_nd_kernel<<<gj, 128, 0, s>>>(ks, nv, b->ml, b->me, ipow_host(q, k - 1) * q, k - 1, b->gr, b->grm,
                                                 b->grw, b->bsp, b->bsq, tmp, 1);
            moments_combine_kernel<<<gj, 128, 0, s>>>(nj, (double)(k + 2), 0, rkd3, tmp);
        }
    }
    if (rkd4) {
        moments_nd_kernel<<<gj, 128, 0, s>>>(ks, nv, b->ml, b->me, ipow_host(q, -(k + 3)), -(k + 3), b->gr, b->grm,
                                             b->grw, b->bsp, b->bsq, rkd4, 0);
        if (mode) {
            moments_nd_kernel<<<gj, 128, 0, s>>>(ks, nv, b->ml, b->me, ipow_host(q, -(k + 4)) * q, -(k + 4), b->gr,
                                                 b->grm, b->grw, b->bsp, b->bsq, tmp, 1);
            moments_combine_kernel<<<gj, 128, 0, s>>>(nj, (double)(k + 1), 1, rkd4, tmp);
        }
    }
    if (rkd) {
        const size_t shm = sizeof(double) * (4 * (size_t)ks * ks * ks + 2 * (size_t)ks * ks);
        if (shm > 48 * 1024) {
            cudaError_t e = smem_attr(vk_diag_cell_kernel, (int)shm);
            if (e != cudaSuccess) return cuda_fail(e, "vk diag_cell smem");
        }
        vk_diag_cell_kernel<<<nv, 256, shm, s>>>(ks, nv, b->ml, b->me, b->h + 1.0, k, mode, b->t, rule_of(b), b->gr,
                                                b->grm, b->grw, b->bsp, b->bsq, b->bspd, rkd);
    }
    return cuda_fail(cudaGetLastError(), mode == 2 ? "qk_moments" : mode ? "wk_moments" : "vk_moments");
}

int launch_mqk_cell(const bsrg_basis *b, const double *rkd1, const double *rkd2, const double *rkd3,
                    const double *rkd4, const double *rkd, double fine, double *rkb, int ldp, cudaStream_t s)
{
    const size_t n = (size_t)b->ns * b->ns * ldp * ldp;
    qkb_expand_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(b->ks, b->ns, b->nv, ldp, fine, rkd1, rkd2, rkd3,
                                                                  rkd4, rkd, rkb);
    return cuda_fail(cudaGetLastError(), "mqk_cell");
}

int launch_mvk_cell(const bsrg_basis *b, const double *rkd1, const double *rkd2, const double *rkd3,
                    const double *rkd4, const double *rkd, double fine, double *rkb, int ldp, cudaStream_t s)
{
    dim3 blk(EXP_TI, EXP_TJ);
    dim3 grd((b->ns + EXP_TI - 1) / EXP_TI, (b->ns + EXP_TJ - 1) / EXP_TJ, ldp * ldp);
    const size_t shm = sizeof(double) * 2 * (size_t)b->ks * ((EXP_TI + b->ks - 1) + (EXP_TJ + b->ks - 1));
    vkb_expand_kernel<<<grd, blk, shm, s>>>(b->ks, b->ns, b->nv, ldp, fine, rkd1, rkd2, rkd3, rkd4, rkd, rkb);
    return cuda_fail(cudaGetLastError(), "mvk_cell");
}

}  // namespace bsrg
