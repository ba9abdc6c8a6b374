// Symmetric tridiagonal eigensolver (divide and conquer) for sm_100a.
//
// The reference's DSYEV (LAP_DSYEV, src/libs/ZCOM/LAPACK_calls.f90:54-76,
// called from diag_hd.f90:312) reduces A to a tridiagonal T and diagonalises T
// by the implicit QL/QR algorithm (DSTEQR).  Here T is diagonalised by Cuppen's
// divide and conquer as in LAPACK's DSTEDC (the published algorithm; Gu and
// Eisenstat's recomputed z for orthogonal eigenvectors), laid out for the GPU:
//
//   * the tree is cut top-down into halves until the pieces have at most
//     DC_LEAF rows; every cut (s, m, e) tears T into T1 (+) T2 + |b| v v^T with
//     b = e(m-1), v = e_{m-1} + sign(b) e_m (the diagonal of both halves loses
//     |b| at the cut);
//   * leaves: one CTA each, cyclic Jacobi with tournament ordering on the dense
//     leaf in shared memory;
//   * merges, one tree level at a time, deepest first: per merge one CTA sorts
//     the poles, finds the tolerance and runs the (sequential) deflation pass
//     -- small z components and close poles merged by a Givens rotation --
//     and lays the surviving columns out by type (upper half only, mixed, lower
//     half only, deflated); the secular equation
//     1 + rho sum z_i^2 / (d_i - lambda) = 0 is solved per root (bracketed
//     Newton, every iterate kept inside a bisection bracket, roots stored as
//     pole + offset); z is recomputed from the roots (Loewner's formula) and
//     the eigenvectors of D + rho z z^T formed column by column; two FP64
//     tensor-core GEMMs per merge (the rows of each half against its column
//     types) give the merged eigenvectors, and a final pass writes eigenvalues
//     and columns in ascending order.
//   The per-level deflation counts are read back to the host once per level
//   (they size the GEMMs).
#include <algorithm>
#include <cmath>
#include <vector>

#include "ctx.h"
#include "dgemm.h"

namespace bsrg {
namespace {

constexpr int DC_LEAF = 64;
constexpr int DC_MAXK = 10240;   // largest merge (shared-memory deflation pass)

struct DcMerge {
    int s, k1, k2, pad;
    long off_g;     // Qg (k x k): gathered child columns, type-grouped, rotations applied
    long off_t;     // Qt (k x k): merged eigenvectors of the non-deflated part
    long off_u;     // U (k x k): eigenvectors of D + rho z z^T (rows in Qg column order)
    long off_v;     // per-merge vectors (8k doubles)
    long off_i;     // per-merge int vectors (4k ints)
};

// per-merge scalars (ints): K, n1, n2, n3, nrot
constexpr int DC_NS = 8;

// ---------------------------------------------------------------------------
// tears and leaves
// ---------------------------------------------------------------------------
__global__ void dc_tear_kernel(int nsplit, const int *__restrict__ splits, double *d, const double *__restrict__ e)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nsplit) return;
    const int m = splits[q];
    const double b = fabs(e[m - 1]);
    d[m - 1] -= b;
    d[m] -= b;
}

// Cyclic Jacobi on one leaf (k <= DC_LEAF), tournament ordering: every round
// rotates k/2 disjoint pairs, rows first, then columns (and V).  Eigenvalues are
// written ascending to w[s..s+k), eigenvectors to Z[s.., s..].
__global__ void __launch_bounds__(256) dc_leaf_kernel(const int *__restrict__ ls, const int *__restrict__ lk,
                                                      const double *__restrict__ d, const double *__restrict__ e,
                                                      double *w, double *Z, long ldz)
{
    extern __shared__ __align__(16) double leaf_sm[];
    double (*A)[DC_LEAF + 1] = (double (*)[DC_LEAF + 1])leaf_sm;
    double (*V)[DC_LEAF + 1] = (double (*)[DC_LEAF + 1])(leaf_sm + DC_LEAF * (DC_LEAF + 1));
    __shared__ double rc[DC_LEAF / 2], rs[DC_LEAF / 2];
    __shared__ int rp[DC_LEAF / 2], rq[DC_LEAF / 2];
    __shared__ int rotated;
    __shared__ int rank[DC_LEAF];
    const int s = ls[blockIdx.x], k = lk[blockIdx.x], tid = threadIdx.x;
    for (int q = tid; q < DC_LEAF * DC_LEAF; q += blockDim.x) {
        const int r = q % DC_LEAF, c = q / DC_LEAF;
        double a = 0.0;
        if (r < k && c < k) {
            if (r == c) a = d[s + r];
            else if (r == c + 1) a = e[s + c];
            else if (c == r + 1) a = e[s + r];
        }
        A[r][c] = a;
        V[r][c] = (r == c) ? 1.0 : 0.0;
    }
    const int m = k + (k & 1);
    const double eps = 2.220446049250313e-16;
    __syncthreads();
    for (int sweep = 0; sweep < 40 && m > 1; sweep++) {
        if (tid == 0) rotated = 0;
        __syncthreads();
        for (int r = 0; r < m - 1; r++) {
            if (tid < m / 2) {
                int p, q;
                if (tid == 0) { p = 0; q = 1 + r % (m - 1); }
                else { p = 1 + (tid + r) % (m - 1); q = 1 + (m - 1 - tid + r) % (m - 1); }
                if (p > q) { int t = p; p = q; q = t; }
                double c = 1.0, sn = 0.0;
                bool act = false;
                if (q < k) {
                    const double apq = A[p][q], app = A[p][p], aqq = A[q][q];
                    if (apq != 0.0 && fabs(apq) > eps * sqrt(fabs(app * aqq))) {
                        const double tau = (aqq - app) / (2.0 * apq);
                        const double t = tau >= 0.0 ? 1.0 / (tau + sqrt(1.0 + tau * tau))
                                                    : -1.0 / (-tau + sqrt(1.0 + tau * tau));
                        c = 1.0 / sqrt(1.0 + t * t);
                        sn = t * c;
                        act = true;
                    }
                }
                rp[tid] = p; rq[tid] = q; rc[tid] = c; rs[tid] = act ? sn : 0.0;
                if (act) rotated = 1;
            }
            __syncthreads();
            // rows p, q of A
            for (int x = tid; x < (m / 2) * k; x += blockDim.x) {
                const int pi = x / k, col = x % k;
                if (rs[pi] == 0.0) continue;
                const int p = rp[pi], q = rq[pi];
                const double c = rc[pi], sn = rs[pi];
                const double ap = A[p][col], aq = A[q][col];
                A[p][col] = c * ap - sn * aq;
                A[q][col] = sn * ap + c * aq;
            }
            __syncthreads();
            // columns p, q of A and V
            for (int x = tid; x < (m / 2) * k; x += blockDim.x) {
                const int pi = x / k, row = x % k;
                if (rs[pi] == 0.0) continue;
                const int p = rp[pi], q = rq[pi];
                const double c = rc[pi], sn = rs[pi];
                const double ap = A[row][p], aq = A[row][q];
                A[row][p] = c * ap - sn * aq;
                A[row][q] = sn * ap + c * aq;
                const double vp = V[row][p], vq = V[row][q];
                V[row][p] = c * vp - sn * vq;
                V[row][q] = sn * vp + c * vq;
            }
            __syncthreads();
        }
        if (!rotated) break;
        __syncthreads();
    }
    // ascending order: rank by value, ties by index
    if (tid < k) {
        const double v = A[tid][tid];
        int rk = 0;
        for (int j = 0; j < k; j++) {
            const double u = A[j][j];
            rk += (u < v) || (u == v && j < tid);
        }
        rank[tid] = rk;
        w[s + rk] = v;
    }
    __syncthreads();
    for (int q = tid; q < k * k; q += blockDim.x) {
        const int r = q % k, c = q / k;
        Z[(s + r) + ldz * (long)(s + rank[c])] = V[r][c];
    }
}

// ---------------------------------------------------------------------------
// merge step 1: sort, deflate, gather the columns (one CTA per merge)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double blk_max(double v, double *sh)
{
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    double r = 0.0;
    for (int q = 0; q < (int)(blockDim.x + 31) / 32; q++) r = fmax(r, sh[q]);
    __syncthreads();
    return r;
}

// Shared layout (dynamic): dS[k] zS[k] (doubles), src[k] (int: child column), st[k] (char:
// 0 deflated, 1 upper, 2 mixed, 3 lower).  Outputs in the merge's vectors:
//   V: dd[K] poles ascending | zz[K] | dval[nd] deflated eigenvalues
//   I: pos[K] Qg column of pole i | gsrc[k] child column of Qg column t | rot (pairs of Qg columns) ...
__global__ void __launch_bounds__(512) dc_prep_kernel(const DcMerge *__restrict__ mg, const double *__restrict__ e,
                                                      const double *__restrict__ w, const double *__restrict__ Z,
                                                      long ldz, double *ws, int *iws, int *scal)
{
    extern __shared__ __align__(16) unsigned char dsm[];
    __shared__ double red[32];
    __shared__ double s_rho;
    __shared__ int s_cnt[4];
    const DcMerge M = mg[blockIdx.x];
    const int k1 = M.k1, k = M.k1 + M.k2, s = M.s, tid = threadIdx.x, nt = blockDim.x;
    double *dS = (double *)dsm, *zS = dS + k;
    int *src = (int *)(zS + k);
    unsigned char *st = (unsigned char *)(src + k);
    double *V = ws + M.off_v;
    double *dd = V, *zz = V + k, *dval = V + 2 * k, *rotc = V + 3 * k, *rots = V + 4 * k;
    int *I = iws + M.off_i;
    int *pos = I, *gsrc = I + k, *rotp = I + 2 * k, *rotq = I + 3 * k;
    int *sc = scal + DC_NS * blockIdx.x;
    const double beta = e[s + k1 - 1];
    const double sg = beta >= 0.0 ? 1.0 : -1.0;
    const double rsq2 = 0.70710678118654752440;
    // merge the two ascending runs (stable: run 1 first on ties)
    for (int i = tid; i < k; i += nt) {
        double v;
        int rk;
        if (i < k1) {
            v = w[s + i];
            int lo = 0, hi = M.k2;   // count run-2 values < v
            while (lo < hi) { int md = (lo + hi) >> 1; if (w[s + k1 + md] < v) lo = md + 1; else hi = md; }
            rk = i + lo;
        } else {
            const int j = i - k1;
            v = w[s + i];
            int lo = 0, hi = k1;     // count run-1 values <= v
            while (lo < hi) { int md = (lo + hi) >> 1; if (w[s + md] <= v) lo = md + 1; else hi = md; }
            rk = j + lo;
        }
        const double zv = i < k1 ? Z[(s + k1 - 1) + ldz * (long)(s + i)] * rsq2
                                 : sg * Z[(s + k1) + ldz * (long)(s + i)] * rsq2;
        dS[rk] = v;
        zS[rk] = zv;
        src[rk] = i;
        st[rk] = i < k1 ? 1 : 3;
    }
    __syncthreads();
    double md = 0.0, mz = 0.0;
    for (int i = tid; i < k; i += nt) { md = fmax(md, fabs(dS[i])); mz = fmax(mz, fabs(zS[i])); }
    md = blk_max(md, red);
    mz = blk_max(mz, red);
    if (tid == 0) {
        const double rho = 2.0 * fabs(beta);
        const double tol = 8.0 * 2.220446049250313e-16 * fmax(md, mz);
        s_rho = rho;
        int nrot = 0;
        if (rho * mz <= tol) {
            for (int i = 0; i < k; i++) st[i] = 0;   // all deflate
        } else {
            int prev = -1;
            for (int j = 0; j < k; j++) {
                if (rho * fabs(zS[j]) <= tol) { st[j] = 0; continue; }
                if (prev >= 0) {
                    const double sv = zS[prev], cv = zS[j];
                    const double tau = hypot(cv, sv);
                    const double t = dS[j] - dS[prev];
                    const double c = cv / tau, sn = -sv / tau;
                    if (fabs(t * c * sn) <= tol) {
                        zS[j] = tau;
                        zS[prev] = 0.0;
                        const int ty = (st[prev] == st[j]) ? st[j] : 2;
                        st[j] = (unsigned char)ty;
                        st[prev] = 0;
                        const double tp = dS[prev] * c * c + dS[j] * sn * sn;
                        dS[j] = dS[prev] * sn * sn + dS[j] * c * c;
                        dS[prev] = tp;
                        // remember: columns (prev, j) rotated by (c, sn); indices mapped to Qg later
                        rotp[nrot] = prev;
                        rotq[nrot] = j;
                        rotc[nrot] = c;
                        rots[nrot] = sn;
                        nrot++;
                    }
                }
                prev = j;
            }
        }
        int n1 = 0, n2 = 0, n3 = 0;
        for (int i = 0; i < k; i++) { n1 += st[i] == 1; n2 += st[i] == 2; n3 += st[i] == 3; }
        s_cnt[0] = n1; s_cnt[1] = n2; s_cnt[2] = n3; s_cnt[3] = nrot;
        sc[0] = n1 + n2 + n3; sc[1] = n1; sc[2] = n2; sc[3] = n3; sc[4] = nrot;
    }
    __syncthreads();
    const int n1 = s_cnt[0], n2 = s_cnt[1], n3 = s_cnt[2];
    const int K = n1 + n2 + n3;
    // Qg column of each sorted position: by type, ascending within each type; poles in
    // ascending order of (rotated) value; deflated last.  One thread, O(k).
    if (tid == 0) {
        // poles (ascending: the rotations can only leave tol-close neighbours out of
        // order, so insertion restores it in ~O(k)) with their Qg column by type;
        // deflated values likewise sorted, their columns after the K pole columns
        int *dpos = I + 5 * k;          // sorted position of each deflated value (temporary)
        int c1 = 0, c2 = n1, c3 = n1 + n2, ip = 0, nd = 0;
        for (int i = 0; i < k; i++) {
            if (st[i] != 0) {
                const int col = st[i] == 1 ? c1++ : (st[i] == 2 ? c2++ : c3++);
                gsrc[col] = i;             // sorted position feeding Qg column col
                int q = ip++;
                while (q > 0 && dd[q - 1] > dS[i]) { dd[q] = dd[q - 1]; zz[q] = zz[q - 1]; pos[q] = pos[q - 1]; q--; }
                dd[q] = dS[i]; zz[q] = zS[i]; pos[q] = col;
            } else {
                int q = nd++;
                while (q > 0 && dval[q - 1] > dS[i]) { dval[q] = dval[q - 1]; dpos[q] = dpos[q - 1]; q--; }
                dval[q] = dS[i]; dpos[q] = i;
            }
        }
        for (int q = 0; q < nd; q++) gsrc[K + q] = dpos[q];
    }
    __syncthreads();
    // rotations recorded on sorted positions -> on Qg columns; child column of every Qg
    // column for the gather (int slab 5k..6k; the deflated-position temporary is done)
    int *colof = (int *)dS;       // dS has been copied out
    for (int c = tid; c < k; c += nt) colof[gsrc[c]] = c;
    __syncthreads();
    for (int t = tid; t < s_cnt[3]; t += nt) { rotp[t] = colof[rotp[t]]; rotq[t] = colof[rotq[t]]; }
    for (int c = tid; c < k; c += nt) I[5 * k + c] = src[gsrc[c]];
    if (tid == 0) {
        double *pr = ws + M.off_v + 7 * (long)k;
        pr[0] = s_rho;
    }
}

// Qg(:, c) = child column feeding Qg column c (zero outside its half).  Threads run
// along rows (coalesced), each covering 32 columns.
__global__ void dc_gather_kernel(const DcMerge *__restrict__ mg, const double *__restrict__ Z, long ldz, double *ws,
                                 const int *__restrict__ iws)
{
    const DcMerge M = mg[blockIdx.z];
    const int k1 = M.k1, k = M.k1 + M.k2, s = M.s;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= k) return;
    const int c0 = blockIdx.y * 32;
    if (c0 >= k) return;
    const int *chcol = iws + M.off_i + 5 * (long)k;
    double *Qg = ws + M.off_g;
    const int c1 = min(c0 + 32, k);
    for (int c = c0; c < c1; c++) {
        const int sc = chcol[c];
        double v = 0.0;
        if ((sc < k1) == (r < k1)) v = Z[(s + r) + ldz * (long)(s + sc)];
        Qg[r + (long)k * c] = v;
    }
}

// the deflation rotations, in order, on every row of Qg (rows are independent)
__global__ void dc_rotate_kernel(const DcMerge *__restrict__ mg, const int *__restrict__ scal, double *ws,
                                 const int *__restrict__ iws)
{
    const DcMerge M = mg[blockIdx.y];
    const int k = M.k1 + M.k2;
    const int nrot = scal[DC_NS * blockIdx.y + 4];
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= k || nrot == 0) return;
    const double *V = ws + M.off_v;
    const double *rotc = V + 3 * (long)k, *rots = V + 4 * (long)k;
    const int *rotp = iws + M.off_i + 2 * (long)k, *rotq = iws + M.off_i + 3 * (long)k;
    double *Qg = ws + M.off_g;
    for (int t = 0; t < nrot; t++) {
        const long a = rotp[t], b = rotq[t];
        const double c = rotc[t], sn = rots[t];
        const double x = Qg[r + k * a], y = Qg[r + k * b];
        Qg[r + k * a] = c * x + sn * y;
        Qg[r + k * b] = c * y - sn * x;
    }
}

// ---------------------------------------------------------------------------
// merge step 2: secular equation, one thread per root
// ---------------------------------------------------------------------------
// root j in (dd_j, dd_{j+1}) (the last in (dd_K, dd_K + rho |z|^2)) as origin index + offset
constexpr int SEC_WARPS = 16;          // roots per CTA of the secular kernel (a warp each)

__device__ __forceinline__ double warp_sum(double x)
{
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

// one warp per root: the lanes split the sums over the poles, every lane then takes the same step
__global__ void __launch_bounds__(32 * SEC_WARPS) dc_secular_kernel(const DcMerge *__restrict__ mg,
                                                                    const int *__restrict__ scal, double *ws,
                                                                    int *iws, int kcap)
{
    extern __shared__ __align__(16) double sm2[];
    const int mi = blockIdx.y;
    const DcMerge M = mg[mi];
    const int k = M.k1 + M.k2;
    const int K = scal[DC_NS * mi];
    if ((int)blockIdx.x * SEC_WARPS >= K) return;
    double *V = ws + M.off_v;
    const double *dd = V, *zz = V + k;
    double *tau = V + 5 * (long)k;
    int *org = iws + M.off_i + 4 * (long)k;
    const double rho = V[7 * (long)k];
    double *sd = sm2, *sz = sm2 + kcap;
    for (int i = threadIdx.x; i < K; i += blockDim.x) { sd[i] = dd[i]; sz[i] = zz[i] * zz[i]; }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int j = blockIdx.x * SEC_WARPS + (threadIdx.x >> 5);
    if (j >= K) return;
    int o;
    double lo, hi;
    if (j < K - 1) {
        const double mid = 0.5 * (sd[j + 1] - sd[j]);
        double fp = 0.0;
        for (int i = lane; i < K; i += 32) fp += sz[i] / ((sd[i] - sd[j]) - mid);
        const double f = 1.0 + rho * warp_sum(fp);
        if (f >= 0.0) { o = j; lo = 0.0; hi = mid; }
        else { o = j + 1; lo = -mid; hi = 0.0; }
    } else {
        double zp = 0.0;
        for (int i = lane; i < K; i += 32) zp += sz[i];
        o = j; lo = 0.0; hi = rho * warp_sum(zp);
    }
    const double dov = sd[o];
    // Iterate on tau with the two-pole model of the secular function (the "middle way" of
    // R.-C. Li, 1993, as LAPACK dlaed4 uses it): psi (poles up to j) and phi (poles above j)
    // are each replaced by a constant plus their nearest pole, matched in value and slope;
    // the model's root in the bracket is the next iterate (the last root: one pole).  Every
    // iterate stays inside [lo, hi]; a step that would leave it bisects instead.
    double t = 0.5 * (lo + hi);
    const double dj = sd[j] - dov, dj1 = j < K - 1 ? sd[j + 1] - dov : 0.0;
    for (int it = 0; it < 100; it++) {
        double psi = 0.0, dpsi = 0.0, phi = 0.0, dphi = 0.0;
        for (int i = lane; i < K; i += 32) {
            const double r = 1.0 / ((sd[i] - dov) - t);
            const double q = sz[i] * r;
            if (i <= j) { psi += q; dpsi += q * r; }
            else { phi += q; dphi += q * r; }
        }
        psi = warp_sum(psi);
        dpsi = warp_sum(dpsi);
        phi = warp_sum(phi);
        dphi = warp_sum(dphi);
        const double eabs = 1.0 + rho * (fabs(psi) + fabs(phi));
        const double f = 1.0 + rho * (psi + phi);
        if (f < 0.0) lo = t; else hi = t;
        if (f == 0.0 || fabs(f) <= 8.0 * 2.220446049250313e-16 * K * eabs) break;
        const double Dj = dj - t;                      // distances to the two nearest poles
        double eta;
        if (j < K - 1) {
            const double Dj1 = dj1 - t;
            const double sj = rho * dpsi * Dj * Dj, sj1 = rho * dphi * Dj1 * Dj1;
            const double c = f - sj / Dj - sj1 / Dj1;
            // c eta^2 - (c (Dj + Dj1) + sj + sj1) eta + (c Dj Dj1 + sj Dj1 + sj1 Dj) = 0
            const double qa = c, qb = c * (Dj + Dj1) + sj + sj1, qc = c * Dj * Dj1 + sj * Dj1 + sj1 * Dj;
            // the model's root between the two poles, eta in (Dj, Dj1); both roots formed stably
            eta = 0.5 * (lo + hi) - t;
            if (qa == 0.0) {
                if (qb != 0.0) eta = qc / qb;
            } else {
                const double disc = sqrt(fmax(qb * qb - 4.0 * qa * qc, 0.0));
                const double w1 = 0.5 * (qb + copysign(disc, qb));
                const double e1 = w1 / qa, e2 = w1 != 0.0 ? qc / w1 : e1;
                if (e1 > Dj && e1 < Dj1) eta = e1;
                else if (e2 > Dj && e2 < Dj1) eta = e2;
            }
        } else {
            const double sj = rho * dpsi * Dj * Dj, c = f - sj / Dj;
            eta = c != 0.0 ? Dj + sj / c : 0.5 * (hi - t);
        }
        double tn = t + eta;
        if (!(tn > lo && tn < hi)) tn = 0.5 * (lo + hi);
        const double step = fabs(tn - t);
        t = tn;
        if (step <= 2.220446049250313e-16 * fabs(t) || hi - lo <= 2.220446049250313e-16 * fmax(fabs(lo), fabs(hi)))
            break;
    }
    if (lane == 0) {
        tau[j] = t;
        org[j] = o;
    }
}

// ---------------------------------------------------------------------------
// merge step 3: z recomputed from the roots, then the eigenvectors of D + rho z z^T
// ---------------------------------------------------------------------------
__global__ void dc_zhat_kernel(const DcMerge *__restrict__ mg, const int *__restrict__ scal, double *ws, int *iws)
{
    const int mi = blockIdx.y;
    const DcMerge M = mg[mi];
    const int k = M.k1 + M.k2;
    const int K = scal[DC_NS * mi];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= K) return;
    double *V = ws + M.off_v;
    const double *dd = V, *zz = V + k, *tau = V + 5 * (long)k;
    double *zh = V + 6 * (long)k;
    const int *org = iws + M.off_i + 4 * (long)k;
    const double di = dd[i];
    // (d_i - lambda_i) prod_{j != i} (d_i - lambda_j) / (d_i - d_j)   (< 0)
    double p = (di - dd[org[i]]) - tau[i];
    for (int j = 0; j < K; j++) {
        if (j == i) continue;
        p *= ((di - dd[org[j]]) - tau[j]) / (di - dd[j]);
    }
    zh[i] = copysign(sqrt(fmax(-p, 0.0)), zz[i]);
}

// U(pos[i], j) = zh_i / (d_i - lambda_j) / ||.||; one warp per column j
__global__ void dc_vec_kernel(const DcMerge *__restrict__ mg, const int *__restrict__ scal, double *ws, int *iws)
{
    const int mi = blockIdx.y;
    const DcMerge M = mg[mi];
    const int k = M.k1 + M.k2;
    const int K = scal[DC_NS * mi];
    const int lane = threadIdx.x & 31;
    const int j = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    if (j >= K) return;
    double *V = ws + M.off_v;
    const double *dd = V, *tau = V + 5 * (long)k, *zh = V + 6 * (long)k;
    const int *pos = iws + M.off_i;
    const int *org = iws + M.off_i + 4 * (long)k;
    double *U = ws + M.off_u;
    const double dj = dd[org[j]], tj = tau[j];
    double ss = 0.0;
    for (int i = lane; i < K; i += 32) {
        const double u = zh[i] / ((dd[i] - dj) - tj);
        ss += u * u;
    }
    for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
    const double inv = 1.0 / sqrt(ss);
    for (int i = lane; i < K; i += 32) {
        const double u = zh[i] / ((dd[i] - dj) - tj);
        U[pos[i] + (long)K * j] = u * inv;
    }
}

// ---------------------------------------------------------------------------
// merge step 4: ascending order of the merged eigenvalues, columns into Z
// ---------------------------------------------------------------------------
// colmap[c] = final column of merged column c (c < K: root c, c >= K: deflated Qg column c)
__global__ void __launch_bounds__(256) dc_rank_kernel(const DcMerge *__restrict__ mg, const int *__restrict__ scal,
                                                      double *ws, int *iws, double *w)
{
    const int mi = blockIdx.x;
    const DcMerge M = mg[mi];
    const int k = M.k1 + M.k2, s = M.s;
    const int K = scal[DC_NS * mi];
    double *V = ws + M.off_v;
    const double *dd = V, *dval = V + 2 * (long)k, *tau = V + 5 * (long)k;
    const int *org = iws + M.off_i + 4 * (long)k;
    int *colmap = iws + M.off_i + 5 * (long)k;
    const int nd = k - K;
    // roots ascending, deflated values ascending: merge by binary search (ties: roots first)
    for (int c = threadIdx.x; c < k; c += blockDim.x) {
        double v;
        int rk;
        if (c < K) {
            v = dd[org[c]] + tau[c];
            int lo = 0, hi = nd;          // deflated values < v
            while (lo < hi) { const int md = (lo + hi) >> 1; if (dval[md] < v) lo = md + 1; else hi = md; }
            rk = c + lo;
        } else {
            const int q = c - K;
            v = dval[q];
            int lo = 0, hi = K;           // roots <= v
            while (lo < hi) {
                const int md = (lo + hi) >> 1;
                if (dd[org[md]] + tau[md] <= v) lo = md + 1; else hi = md;
            }
            rk = q + lo;
        }
        colmap[c] = rk;
        w[s + rk] = v;
    }
}

__global__ void dc_copy_kernel(const DcMerge *__restrict__ mg, const int *__restrict__ scal, const double *ws,
                               const int *iws, double *Z, long ldz)
{
    const int mi = blockIdx.y;
    const DcMerge M = mg[mi];
    const int k = M.k1 + M.k2, s = M.s;
    const int K = scal[DC_NS * mi];
    const int *colmap = iws + M.off_i + 5 * (long)k;
    const double *Qt = ws + M.off_t, *Qg = ws + M.off_g;
    for (int c = blockIdx.x; c < k; c += gridDim.x) {
        const double *src = c < K ? Qt + (long)k * c : Qg + (long)k * c;
        double *dst = Z + s + ldz * (long)(s + colmap[c]);
        for (int r = threadIdx.x; r < k; r += blockDim.x) dst[r] = src[r];
    }
}

struct Node { int s, k1, k2; };

}  // namespace

size_t dc_workspace_bytes(int n)
{
    // per level: sum over merges of 3k^2 + 8k doubles and 6k ints, at most 3n^2 + 8n doubles
    const size_t dbl = 3 * (size_t)n * n + 8 * (size_t)n + 64;
    const size_t ints = 6 * (size_t)n + 64;
    const size_t maxm = (size_t)n / (DC_LEAF / 2) + 8;
    // splits, leaf starts and sizes, merge descriptors, per-merge scalars, 256-byte alignment of 7 parts
    return dbl * 8 + ints * 4 + maxm * (3 * sizeof(int) + sizeof(DcMerge) + DC_NS * sizeof(int)) + 8 * 256 + 1024;
}

// T = tridiag(d, e) (device; d is overwritten by the torn diagonal), eigenvalues
// ascending into w, eigenvectors into Z (ldz).  ws: dc_workspace_bytes(n) device
// bytes; pinned: dc_pinned_bytes(n) bytes of pinned host staging.
size_t dc_pinned_bytes(int n)
{
    const size_t maxm = (size_t)n / (DC_LEAF / 2) + 8;
    return maxm * (3 * sizeof(int) + sizeof(DcMerge) + DC_NS * sizeof(int)) + 256;
}

int tridiag_dc(cudaStream_t st, int n, double *d, const double *e, double *w, double *Z, long ldz, void *ws_base,
               size_t ws_bytes, void *pinned, size_t pinned_bytes, double *gemm_flops, int *launches)
{
    if (gemm_flops) *gemm_flops = 0.0;
    if (launches) *launches = 0;
    if (n < 1) return BSRG_OK;
    int nlaunch = 0;
    if (n > DC_MAXK) { set_error("dstedc: n=%d above %d", n, DC_MAXK); return BSRG_ERR_ARG; }
    if (ws_bytes < dc_workspace_bytes(n) || pinned_bytes < dc_pinned_bytes(n)) {
        set_error("dstedc: workspace too small");
        return BSRG_ERR_NOMEM;
    }
    cudaError_t err;
    // ---- the tree (host): halves down to DC_LEAF rows ----
    std::vector<Node> leaves;                  // s, k1 = size
    std::vector<std::vector<Node>> merges;     // by depth
    std::vector<int> splits;
    struct Frame { int s, n, depth; };
    std::vector<Frame> stack{{0, n, 0}};
    while (!stack.empty()) {
        Frame f = stack.back();
        stack.pop_back();
        if (f.n <= DC_LEAF) { leaves.push_back({f.s, f.n, 0}); continue; }
        const int h = f.n / 2;
        if ((int)merges.size() <= f.depth) merges.resize(f.depth + 1);
        merges[f.depth].push_back({f.s, h, f.n - h});
        splits.push_back(f.s + h);
        stack.push_back({f.s, h, f.depth + 1});
        stack.push_back({f.s + h, f.n - h, f.depth + 1});
    }
    // ---- workspace layout ----
    char *base = (char *)ws_base;
    size_t off = 0;
    auto take = [&](size_t bytes) { off = (off + 255) & ~(size_t)255; char *p = base + off; off += bytes; return p; };
    const size_t maxm = (size_t)n / (DC_LEAF / 2) + 8;
    int *d_splits = (int *)take(sizeof(int) * maxm);
    int *d_ls = (int *)take(sizeof(int) * maxm), *d_lk = (int *)take(sizeof(int) * maxm);
    DcMerge *d_mg = (DcMerge *)take(sizeof(DcMerge) * maxm);
    int *d_scal = (int *)take(sizeof(int) * DC_NS * maxm);
    double *wsd = (double *)take(sizeof(double) * (3 * (size_t)n * n + 8 * (size_t)n + 64));
    int *wsi = (int *)take(sizeof(int) * (6 * (size_t)n + 64));
    if (off > ws_bytes || leaves.size() > maxm || splits.size() > maxm) {
        set_error("dstedc: workspace layout");
        return BSRG_ERR_NOMEM;
    }
    char *pb = (char *)pinned;
    int *h_splits = (int *)pb, *h_ls = h_splits + maxm, *h_lk = h_ls + maxm;
    DcMerge *h_mg = (DcMerge *)(((uintptr_t)(h_lk + maxm) + 15) & ~(uintptr_t)15);
    int *h_scal = (int *)(h_mg + maxm);
    for (size_t q = 0; q < splits.size(); q++) h_splits[q] = splits[q];
    for (size_t q = 0; q < leaves.size(); q++) { h_ls[q] = leaves[q].s; h_lk[q] = leaves[q].k1; }
    if (!splits.empty()) {
        if ((err = cudaMemcpyAsync(d_splits, h_splits, sizeof(int) * splits.size(), cudaMemcpyHostToDevice, st)) !=
            cudaSuccess)
            return cuda_fail(err, "dstedc upload");
        dc_tear_kernel<<<(unsigned)((splits.size() + 127) / 128), 128, 0, st>>>((int)splits.size(), d_splits, d, e);
    }
    if ((err = cudaMemcpyAsync(d_ls, h_ls, sizeof(int) * leaves.size(), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (err = cudaMemcpyAsync(d_lk, h_lk, sizeof(int) * leaves.size(), cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return cuda_fail(err, "dstedc upload");
    const int smem_leaf = 2 * DC_LEAF * (DC_LEAF + 1) * (int)sizeof(double);
    if ((err = smem_attr(dc_leaf_kernel, smem_leaf)) !=
        cudaSuccess)
        return cuda_fail(err, "dstedc leaf smem");
    dc_leaf_kernel<<<(unsigned)leaves.size(), 256, smem_leaf, st>>>(d_ls, d_lk, d, e, w, Z, ldz);
    if ((err = cudaGetLastError()) != cudaSuccess) return cuda_fail(err, "dstedc leaves");
    // ---- merges, deepest level first ----
    for (int lv = (int)merges.size() - 1; lv >= 0; lv--) {
        const std::vector<Node> &L = merges[lv];
        const int nm = (int)L.size();
        long og = 0, ov = 0, oi = 0;
        int kmax = 0;
        for (int q = 0; q < nm; q++) {
            DcMerge &M = h_mg[q];
            const long k = L[q].k1 + L[q].k2;
            M.s = L[q].s; M.k1 = L[q].k1; M.k2 = L[q].k2; M.pad = 0;
            M.off_g = og; og += k * k;
            M.off_t = og; og += k * k;
            M.off_u = og; og += k * k;
            M.off_v = 3 * (long)n * n + ov; ov += 8 * k;
            M.off_i = oi; oi += 6 * k;
            kmax = std::max<int>(kmax, (int)k);
        }
        if ((err = cudaMemcpyAsync(d_mg, h_mg, sizeof(DcMerge) * nm, cudaMemcpyHostToDevice, st)) != cudaSuccess)
            return cuda_fail(err, "dstedc merge upload");
        const int smem_prep = kmax * 21 + 64;
        if ((err = smem_attr(dc_prep_kernel, smem_prep)) !=
            cudaSuccess)
            return cuda_fail(err, "dstedc prep smem");
        dc_prep_kernel<<<nm, 512, smem_prep, st>>>(d_mg, e, w, Z, ldz, wsd, wsi, d_scal);
        if ((err = cudaMemcpyAsync(h_scal, d_scal, sizeof(int) * DC_NS * nm, cudaMemcpyDeviceToHost, st)) !=
                cudaSuccess ||
            (err = cudaStreamSynchronize(st)) != cudaSuccess)
            return cuda_fail(err, "dstedc deflation");
        {
            dim3 gg((unsigned)((kmax + 127) / 128), (unsigned)((kmax + 31) / 32), nm);
            dc_gather_kernel<<<gg, 128, 0, st>>>(d_mg, Z, ldz, wsd, wsi);
            dim3 gr((unsigned)((kmax + 127) / 128), nm);
            dc_rotate_kernel<<<gr, 128, 0, st>>>(d_mg, d_scal, wsd, wsi);
        }
        int Kmax = 0;
        for (int q = 0; q < nm; q++) Kmax = std::max(Kmax, h_scal[DC_NS * q]);
        if (Kmax > 0) {
            const int smem_sec = 16 * Kmax;
            if ((err = smem_attr(dc_secular_kernel, smem_sec)) != cudaSuccess)
                return cuda_fail(err, "dstedc secular smem");
            dim3 gsec((unsigned)((Kmax + SEC_WARPS - 1) / SEC_WARPS), nm);
            dc_secular_kernel<<<gsec, 32 * SEC_WARPS, smem_sec, st>>>(d_mg, d_scal, wsd, wsi, Kmax);
            dim3 gs((unsigned)((Kmax + 127) / 128), nm);
            dc_zhat_kernel<<<gs, 128, 0, st>>>(d_mg, d_scal, wsd, wsi);
            dim3 gv((unsigned)((Kmax + 7) / 8), nm);
            dc_vec_kernel<<<gv, 256, 0, st>>>(d_mg, d_scal, wsd, wsi);
            for (int q = 0; q < nm; q++) {
                const DcMerge &M = h_mg[q];
                const int k = M.k1 + M.k2, K = h_scal[DC_NS * q], n1 = h_scal[DC_NS * q + 1],
                          n2 = h_scal[DC_NS * q + 2];
                if (K == 0) continue;
                const double *Qg = wsd + M.off_g, *U = wsd + M.off_u;
                double *Qt = wsd + M.off_t;
                // upper rows: Q1 columns (types 1, 2); lower rows: types 2, 3
                if (gemm_flops) *gemm_flops += 2.0 * K * ((double)M.k1 * (n1 + n2) + (double)M.k2 * (K - n1));
                nlaunch += 2;
                int rc = dgemm(false, false, M.k1, K, n1 + n2, 1.0, Qg, k, U, K, 0.0, Qt, k, st);
                if (rc == BSRG_OK)
                    rc = dgemm(false, false, M.k2, K, K - n1, 1.0, Qg + M.k1 + (long)k * n1, k, U + n1, K, 0.0,
                               Qt + M.k1, k, st);
                if (rc != BSRG_OK) return rc;
            }
        }
        nlaunch += 3 + (Kmax > 0 ? 3 : 0) + 2;
        dc_rank_kernel<<<nm, 256, 0, st>>>(d_mg, d_scal, wsd, wsi, w);
        dim3 gc((unsigned)std::min(kmax, 2048), nm);
        dc_copy_kernel<<<gc, 128, 0, st>>>(d_mg, d_scal, wsd, wsi, Z, ldz);
        if ((err = cudaGetLastError()) != cudaSuccess) return cuda_fail(err, "dstedc merge");
    }
    if (launches) *launches = nlaunch + 2;
    return BSRG_OK;
}

}  // namespace bsrg

using namespace bsrg;

extern "C" int bsrg_dstedc(bsrg_ctx *c, int n, const double *d, const double *e, double *w, double *Z, int ldz)
{
    if (!c || (n > 0 && (!d || !w || !Z || (n > 1 && !e)))) { set_error("dstedc: null argument"); return BSRG_ERR_ARG; }
    if (n < 0 || ldz < (n > 0 ? n : 1)) { set_error("dstedc: n=%d ldz=%d", n, ldz); return BSRG_ERR_ARG; }
    if (n == 0) return BSRG_OK;
    cudaSetDevice(c->device);
    const size_t need = dc_workspace_bytes(n) + sizeof(double) * (size_t)n + 1024;
    int rc = ctx_reserve(c, need);
    if (rc == BSRG_OK) rc = ctx_reserve_pinned(c, dc_pinned_bytes(n));
    if (rc != BSRG_OK) return rc;
    cudaStream_t s = c->stream;
    double *dt = (double *)c->ws;                        // torn copy of d
    char *rest = (char *)c->ws + (((size_t)n * sizeof(double) + 255) & ~(size_t)255);
    cudaError_t e1 = cudaMemcpyAsync(dt, d, sizeof(double) * n, cudaMemcpyDeviceToDevice, s);
    if (e1 != cudaSuccess) return cuda_fail(e1, "dstedc copy");
    static const double zero = 0.0;
    rc = tridiag_dc(s, n, dt, n > 1 ? e : &zero, w, Z, ldz, rest, c->ws_bytes - (rest - (char *)c->ws), c->pinned,
                    c->pinned_bytes, nullptr, nullptr);
    if (rc != BSRG_OK) return rc;
    cudaEventRecord(c->ev_stage, s);
    return cuda_fail(cudaGetLastError(), "dstedc");
}
