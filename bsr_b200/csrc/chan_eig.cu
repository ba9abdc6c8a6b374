// The channel eigenproblems of diag_hd as the library's own batched kernels.
//
// Reference: src/bsr/BSR_HD3/diag_hd.f90:82-111 -- for every channel, LAPACK
// DSYGV('V','U') of (H_ii, S_ii) restricted to the splines l+2..ns (or ns-1).
// Here, with one CTA per channel for every step (40 channels of n ~ 200 at
// the config-2 size):
//   1. chan_tridiag_kernel: the banded Cholesky S = L L^T (bandwidth ks), the
//      reduction C = L^-1 H L^-T by banded substitutions, and the Householder
//      tridiagonalisation of C (LAPACK dsytd2's lower-triangle convention:
//      C = Q T Q^T, Q = H_0 H_1 ... H_{n-3}) on C packed in shared memory;
//   2. chan_eigvec_kernel: every eigenvalue of T by bisection on Sturm counts
//      (to a relative width of 2 eps, as far as the counts resolve), and its eigenvector
//      by inverse iteration (LU of T - lambda I with partial pivoting, three
//      solves from a fixed pseudo-random start), one thread per eigenpair;
//   3. (host) symmetric orthogonalisation of the eigenvectors, twice:
//      Y <- Y (3/2 I - 1/2 Y^T Y) as batched FP64 tensor-core GEMMs.  Inverse
//      iteration leaves eigenvectors of close eigenvalues non-orthogonal by
//      ~eps ||T|| / gap; mixing y_j with y_i by that amount changes the residual
//      of y_j by ~eps ||T||, so the pairs stay accurate and become orthonormal;
//   4. chan_back_kernel: x = L^-T Q y, panel by panel in shared memory.
// The eigenvectors come out S-orthonormal (x^T S x = 1) in ascending order of
// their eigenvalues, as DSYGV returns them (up to the sign of each vector).
#include <cfloat>

#include "ctx.h"
#include "dgemm.h"

namespace bsrg {

constexpr int CH_THREADS = 256;

__host__ __device__ inline size_t tri(int i) { return (size_t)i * (i + 1) / 2; }

// CTA-wide sum (every thread gets the result); red holds 32 doubles
__device__ inline double cta_sum(double v, double *red)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();                              // red is free (a previous sum has been read)
    if (lane == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); q++) s += red[q];
    return s;
}

// S(i, j) of the channel restricted to rows/columns s0.. (sb: band (ns, ks), lower)
__device__ inline double s_restricted(const double *sb, int ns, int ks, int s0, int i, int j)
{
    const int hi = s0 + (i > j ? i : j), lo = s0 + (i > j ? j : i);
    return hi - lo < ks ? sb[hi + (size_t)ns * (lo - hi + ks - 1)] : 0.0;
}

template <int KS>
__global__ void __launch_bounds__(CH_THREADS)
chan_tridiag_kernel(int ns, int npad, const int *__restrict__ s0v, const int *__restrict__ nsolv,
                    const double *__restrict__ hcc, const double *__restrict__ sb, double *Xg, double *Lg,
                    double *Vg, double *dg, double *eg, double *taug, int *info)
{
    extern __shared__ double cs[];
    const int ich = blockIdx.x, n = nsolv[ich], s0 = s0v[ich];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const size_t np2 = (size_t)npad * npad, npk = tri(npad);
    double *Cp = cs;                          // C, packed lower (row i at tri(i))
    double *Lb = Cp + npk;                    // L band: row i, column j at i*KS + (j - i + KS - 1)
    double *vs = Lb + (size_t)npad * KS;      // reflector
    double *ws = vs + npad;                   // p, then w
    double *es = ws + npad, *ts = es + npad;  // off-diagonal, tau
    double *red = ts + npad;                  // 32 + 1
    int *bad = (int *)(red + 33);
    const double *H = hcc + ((size_t)(ich + 1) * (ich + 2) / 2 - 1) * ns * ns;
    double *X = Xg + (size_t)ich * np2;
    for (int q = tid; q < npad * KS; q += CH_THREADS) Lb[q] = 0.0;
    if (tid == 0) *bad = 0;
    __syncthreads();
    // ---- banded Cholesky (one warp, column by column) ----
    if (w == 0) {
        for (int j = 0; j < n; j++) {
            if (lane == 0) {
                double dsum = s_restricted(sb, ns, KS, s0, j, j);
                for (int k = j - KS + 1 > 0 ? j - KS + 1 : 0; k < j; k++) {
                    const double l = Lb[j * KS + (k - j + KS - 1)];
                    dsum -= l * l;
                }
                if (!(dsum > 0.0)) {         // not positive definite: flagged, kept finite
                    if (*bad == 0) *bad = j + 1;
                    dsum = 1.0;
                }
                Lb[j * KS + KS - 1] = sqrt(dsum);
            }
            __syncwarp();
            const double ljj = Lb[j * KS + KS - 1];
            const int i = j + 1 + lane;
            if (lane < KS - 1 && i < n) {
                double v = s_restricted(sb, ns, KS, s0, i, j);
                for (int k = i - KS + 1 > 0 ? i - KS + 1 : 0; k < j; k++)
                    v -= Lb[i * KS + (k - i + KS - 1)] * Lb[j * KS + (k - j + KS - 1)];
                Lb[i * KS + (j - i + KS - 1)] = v / ljj;
            }
            __syncwarp();
        }
    }
    __syncthreads();
    // ---- X = L^-1 H (thread per column; H symmetric, read along its rows) ----
    for (int c = tid; c < n; c += CH_THREADS) {
        double win[KS];
#pragma unroll
        for (int t = 0; t < KS; t++) win[t] = 0.0;
        const double *Hc = H + (s0 + c);
        for (int i = 0; i < n; i++) {
            double v = Hc[(size_t)ns * (s0 + i)];
#pragma unroll
            for (int t = 1; t < KS; t++)
                if (i - t >= 0) v -= Lb[i * KS + KS - 1 - t] * win[t - 1];
            v /= Lb[i * KS + KS - 1];
#pragma unroll
            for (int t = KS - 2; t > 0; t--) win[t] = win[t - 1];
            win[0] = v;
            X[(size_t)i * npad + c] = v;
        }
    }
    __syncthreads();
    // ---- C = L^-1 X^T, lower triangle packed in shared memory ----
    for (int c = tid; c < n; c += CH_THREADS) {
        double win[KS];
#pragma unroll
        for (int t = 0; t < KS; t++) win[t] = 0.0;
        const double *Xr = X + (size_t)c * npad;      // X(c, i) = X^T(i, c)
        for (int i = 0; i < n; i++) {
            double v = Xr[i];
#pragma unroll
            for (int t = 1; t < KS; t++)
                if (i - t >= 0) v -= Lb[i * KS + KS - 1 - t] * win[t - 1];
            v /= Lb[i * KS + KS - 1];
#pragma unroll
            for (int t = KS - 2; t > 0; t--) win[t] = win[t - 1];
            win[0] = v;
            if (i >= c) Cp[tri(i) + c] = v;
        }
    }
    __syncthreads();
    // ---- Householder tridiagonalisation (dsytd2, lower) ----
    for (int k = 0; k + 2 < n; k++) {
        const int m = n - k - 1;                 // trailing rows k+1 .. n-1
        double part = 0.0;
        for (int i = k + 2 + tid; i < n; i += CH_THREADS) {
            const double x = Cp[tri(i) + k];
            part += x * x;
        }
        const double sigma = cta_sum(part, red);
        const double alpha = Cp[tri(k + 1) + k];
        double tau, beta, scal;
        if (sigma == 0.0) {
            tau = 0.0; beta = alpha; scal = 0.0;
        } else {
            beta = -copysign(sqrt(alpha * alpha + sigma), alpha);
            tau = (beta - alpha) / beta;
            scal = 1.0 / (alpha - beta);
        }
        // v = (1, C(k+2.., k) scal); column k keeps v below its first entry for the back-transform
        for (int r = tid; r < m; r += CH_THREADS) {
            double v = 1.0;
            if (r > 0) {
                v = Cp[tri(k + 1 + r) + k] * scal;
                Cp[tri(k + 1 + r) + k] = v;
            }
            vs[r] = v;
        }
        if (tid == 0) { es[k] = beta; ts[k] = tau; }
        __syncthreads();
        if (tau == 0.0) continue;
        // p = tau C v over the trailing block (thread per row; the row's two halves of the symmetric matrix)
        for (int r = tid; r < m; r += CH_THREADS) {
            const int i = k + 1 + r;
            const double *rowi = Cp + tri(i) + (k + 1);
            double s = 0.0;
            for (int j = 0; j <= r; j++) s = fma(rowi[j], vs[j], s);
            for (int j = r + 1; j < m; j++) s = fma(Cp[tri(k + 1 + j) + i], vs[j], s);
            ws[r] = tau * s;
        }
        __syncthreads();
        part = 0.0;
        for (int r = tid; r < m; r += CH_THREADS) part += ws[r] * vs[r];
        const double gam = -0.5 * tau * cta_sum(part, red);
        for (int r = tid; r < m; r += CH_THREADS) ws[r] = fma(gam, vs[r], ws[r]);
        __syncthreads();
        // C -= v w^T + w v^T on the trailing lower triangle (warp per row)
        for (int r = w; r < m; r += CH_THREADS / 32) {
            const double vi = vs[r], wi = ws[r];
            double *rowi = Cp + tri(k + 1 + r) + (k + 1);
            for (int j = lane; j <= r; j += 32) rowi[j] -= vi * ws[j] + wi * vs[j];
        }
        __syncthreads();
    }
    // ---- outputs: d, e, tau, the reflectors (packed C) and L ----
    double *dgc = dg + (size_t)ich * npad, *egc = eg + (size_t)ich * npad, *tgc = taug + (size_t)ich * npad;
    for (int i = tid; i < n; i += CH_THREADS) {
        dgc[i] = Cp[tri(i) + i];
        if (i + 2 < n) { egc[i] = es[i]; tgc[i] = ts[i]; }
        else if (i + 2 == n) { egc[i] = Cp[tri(n - 1) + n - 2]; tgc[i] = 0.0; }
    }
    double *Vc = Vg + (size_t)ich * npk;
    for (size_t q = tid; q < tri(n); q += CH_THREADS) Vc[q] = Cp[q];
    double *Lc = Lg + (size_t)ich * npad * KS;
    for (int q = tid; q < n * KS; q += CH_THREADS) Lc[q] = Lb[q];
    if (tid == 0) info[ich] = *bad;
}

// pseudo-random start vector entry in [-1, 1) for eigenpair j, row i (a fixed integer hash)
__device__ inline double start_entry(int i, int j)
{
    unsigned h = (unsigned)i * 0x9E3779B1u ^ ((unsigned)j * 0x85EBCA77u + 0xC2B2AE3Du);
    h ^= h >> 15; h *= 0x2C1B3C6Du; h ^= h >> 12; h *= 0x297A2D39u; h ^= h >> 15;
    return (double)h * (2.0 / 4294967296.0) - 1.0;
}

constexpr int CH_NMAX = 1024;      // rows of T a chan_eigvec_kernel CTA stages

// Eigenpair j of channel blockIdx.x's tridiagonal T, j = blockIdx.y*128 + thread.
// Y (row i, column j at Y[i*npad + j], i.e. the transposed eigenvector matrix in
// column-major terms) gets the unit eigenvector, zero outside the n x n block;
// scratch holds the LU factors, five npad x npad arrays per channel.
__global__ void __launch_bounds__(128)
chan_eigvec_kernel(int ns, int npad, const int *__restrict__ nsolv, const double *__restrict__ dg,
                   const double *__restrict__ eg, double *Wv, double *Yg, double *scratch)
{
    __shared__ double d[CH_NMAX], e2[CH_NMAX], e[CH_NMAX];
    const int ich = blockIdx.x, n = nsolv[ich];
    const size_t np2 = (size_t)npad * npad;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        d[i] = dg[(size_t)ich * npad + i];
        const double ei = i + 1 < n ? eg[(size_t)ich * npad + i] : 0.0;
        e[i] = ei;
        e2[i] = ei * ei;
    }
    __syncthreads();
    const int j = blockIdx.y * blockDim.x + threadIdx.x;
    double *Y = Yg + (size_t)ich * np2;
    if (j >= npad) return;
    if (j >= n) {
        for (int i = 0; i < npad; i++) Y[(size_t)i * npad + j] = 0.0;
        return;
    }
    // Gershgorin interval and the pivot floor of the Sturm counts (dstebz)
    double gl = DBL_MAX, gu = -DBL_MAX, emax2 = 0.0;
    for (int i = 0; i < n; i++) {
        const double r = (i > 0 ? fabs(e[i - 1]) : 0.0) + fabs(e[i]);
        gl = fmin(gl, d[i] - r);
        gu = fmax(gu, d[i] + r);
        emax2 = fmax(emax2, e2[i]);
    }
    const double eps = DBL_EPSILON, tnorm = fmax(fabs(gl), fabs(gu));
    const double pivmin = DBL_MIN * fmax(1.0, emax2);
    double lo = gl - 2.0 * eps * tnorm - 2.0 * pivmin, hi = gu + 2.0 * eps * tnorm + 2.0 * pivmin;
    // ---- bisection: the (j+1)-th smallest eigenvalue ----
    for (int it = 0; it < 128; it++) {
        const double mid = 0.5 * (lo + hi);
        if (hi - lo <= 2.0 * eps * fmax(fabs(lo), fabs(hi)) + 2.0 * pivmin || mid <= lo || mid >= hi) break;
        int cnt = 0;
        double q = d[0] - mid;
        if (fabs(q) < pivmin) q = -pivmin;
        cnt += q < 0.0;
        for (int i = 1; i < n; i++) {
            q = (d[i] - mid) - e2[i - 1] / q;
            if (fabs(q) < pivmin) q = -pivmin;
            cnt += q < 0.0;
        }
        if (cnt > j) hi = mid;
        else lo = mid;
    }
    const double lam = 0.5 * (lo + hi);
    Wv[(size_t)ich * ns + j] = lam;
    // ---- LU of T - lam I with partial pivoting (rows i, i+1 at step i) ----
    double *A = scratch + (size_t)ich * 5 * np2, *UP = A + np2, *C2 = UP + np2, *LL = C2 + np2, *PV = LL + np2;
    const double tiny = tnorm > 0.0 ? eps * tnorm : DBL_MIN;
#define AT(arr, i) arr[(size_t)(i) * npad + j]
    double ai = d[0] - lam, ui = n > 1 ? e[0] : 0.0;
    for (int i = 0; i + 1 < n; i++) {
        const double li = e[i], di1 = d[i + 1] - lam, ui1 = i + 2 < n ? e[i + 1] : 0.0;
        double mlt;
        if (fabs(ai) >= fabs(li)) {
            if (ai == 0.0) ai = tiny;
            mlt = li / ai;
            AT(A, i) = ai; AT(UP, i) = ui; AT(C2, i) = 0.0; AT(PV, i) = 0.0;
            ai = di1 - mlt * ui;
            ui = ui1;
        } else {
            mlt = ai / li;
            AT(A, i) = li; AT(UP, i) = di1; AT(C2, i) = ui1; AT(PV, i) = 1.0;
            ai = ui - mlt * di1;
            ui = -mlt * ui1;
        }
        AT(LL, i) = mlt;
    }
    if (ai == 0.0) ai = tiny;
    AT(A, n - 1) = ai;
    // ---- three inverse-iteration solves, normalised; x kept in Y ----
    double scale = 1.0;
    for (int it = 0; it < 3; it++) {
        // forward: y = L^-1 P b, b = the start vector or the previous x * scale
        double yc = it == 0 ? start_entry(0, j) : AT(Y, 0) * scale;
        for (int i = 0; i + 1 < n; i++) {
            const double yn = it == 0 ? start_entry(i + 1, j) : AT(Y, i + 1) * scale;
            const double mlt = AT(LL, i);
            if (AT(PV, i) != 0.0) {
                AT(Y, i) = yn;
                yc = yc - mlt * yn;
            } else {
                AT(Y, i) = yc;
                yc = yn - mlt * yc;
            }
        }
        AT(Y, n - 1) = yc;
        // back: U x = y, U with two superdiagonals
        double x1 = AT(Y, n - 1) / AT(A, n - 1), x2 = 0.0;
        AT(Y, n - 1) = x1;
        double ss = x1 * x1;
        for (int i = n - 2; i >= 0; i--) {
            const double x = (AT(Y, i) - AT(UP, i) * x1 - AT(C2, i) * x2) / AT(A, i);
            AT(Y, i) = x;
            ss += x * x;
            x2 = x1;
            x1 = x;
        }
        scale = 1.0 / sqrt(ss);
    }
    for (int i = 0; i < n; i++) AT(Y, i) *= scale;
    for (int i = n; i < npad; i++) AT(Y, i) = 0.0;
#undef AT
}

// M = 3/2 I - 1/2 G for the symmetric orthogonalisation step; flag if G is far from I
__global__ void chan_lowdin_kernel(int npad, const int *__restrict__ nsolv, double *G, int *flag)
{
    const int ich = blockIdx.y, n = nsolv[ich];
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (size_t)npad * npad) return;
    const int r = (int)(q % npad), c = (int)(q / npad);
    double *g = G + (size_t)ich * npad * npad + q;
    const double id = r == c ? 1.0 : 0.0;
    if (r < n && c < n && fabs(*g - id) > 1e-3) atomicExch(flag, 1);
    *g = 1.5 * id - 0.5 * *g;
}

// x = L^-T Q y for every eigenvector of the channel, panel by panel (pw vectors)
template <int KS>
__global__ void __launch_bounds__(CH_THREADS)
chan_back_kernel(int ns, int npad, int pw, const int *__restrict__ nsolv, const double *__restrict__ Vg,
                 const double *__restrict__ taug, const double *__restrict__ Lg, const double *__restrict__ Yg,
                 double *AA)
{
    extern __shared__ double cs[];
    const int ich = blockIdx.x, n = nsolv[ich], tid = threadIdx.x;
    const size_t np2 = (size_t)npad * npad, npk = tri(npad);
    const int pws = pw + 1;                     // panel row stride
    double *Vp = cs, *tau = Vp + npk, *Lb = tau + npad, *vk = Lb + (size_t)npad * KS, *wc = vk + 2 * (size_t)npad;
    double *red = wc + pw, *Zp = red + CH_THREADS;
    static_assert(CH_THREADS % 32 == 0, "panel widths 8, 16, 32 divide the CTA");
    for (size_t q = tid; q < tri(n); q += CH_THREADS) Vp[q] = Vg[(size_t)ich * npk + q];
    for (int q = tid; q < n; q += CH_THREADS) tau[q] = q + 2 < n ? taug[(size_t)ich * npad + q] : 0.0;
    for (int q = tid; q < n * KS; q += CH_THREADS) Lb[q] = Lg[(size_t)ich * npad * KS + q];
    const double *Y = Yg + (size_t)ich * np2;
    double *X = AA + (size_t)ich * ns * ns;
    const int G = CH_THREADS / pw;               // row groups of the dot products
    for (int j0 = 0; j0 < n; j0 += pw) {
        const int nc = n - j0 < pw ? n - j0 : pw;
        __syncthreads();                         // previous panel written out
        for (int q = tid; q < n * pw; q += CH_THREADS) {
            const int r = q / pw, c = q % pw;
            Zp[r * pws + c] = c < nc ? Y[(size_t)r * npad + j0 + c] : 0.0;
        }
        // reflector n-3 first: Q y = H_0 (H_1 (... H_{n-3} y))
        int cur = 0;
        if (n >= 3) {
            const int k = n - 3, m = n - k - 1;
            for (int r = tid; r < m; r += CH_THREADS) vk[r] = r == 0 ? 1.0 : Vp[tri(k + 1 + r) + k];
        }
        __syncthreads();
        for (int k = n - 3; k >= 0; k--) {
            const int m = n - k - 1;
            const double *v = vk + (size_t)cur * npad;
            const double tk = tau[k];
            if (tk != 0.0) {
                // partial dots of v with the panel's columns
                const int c = tid % pw, g = tid / pw;
                double s = 0.0;
                if (g < G)
                    for (int r = g; r < m; r += G) s = fma(v[r], Zp[(k + 1 + r) * pws + c], s);
                red[tid] = s;
            }
            // the next reflector into the other buffer
            if (k > 0) {
                double *vn = vk + (size_t)(cur ^ 1) * npad;
                const int kn = k - 1, mn = n - kn - 1;
                for (int r = tid; r < mn; r += CH_THREADS) vn[r] = r == 0 ? 1.0 : Vp[tri(kn + 1 + r) + kn];
            }
            __syncthreads();
            if (tk != 0.0) {
                // CH_THREADS is a multiple of pw: a thread updates one column throughout
                const int c = tid % pw;
                double wsum = 0.0;
                for (int g = 0; g < G; g++) wsum += red[g * pw + c];
                wsum *= tk;
                for (int r = tid / pw; r < m; r += G) Zp[(k + 1 + r) * pws + c] -= v[r] * wsum;
            }
            cur ^= 1;
            __syncthreads();
        }
        // x = L^-T z, column by column from the last row
        if (tid < nc) {
            const int c = tid;
            double win[KS];
#pragma unroll
            for (int t = 0; t < KS; t++) win[t] = 0.0;
            for (int i = n - 1; i >= 0; i--) {
                double v = Zp[i * pws + c];
#pragma unroll
                for (int t = 1; t < KS; t++)
                    if (i + t < n) v -= Lb[(i + t) * KS + KS - 1 - t] * win[t - 1];
                v /= Lb[i * KS + KS - 1];
#pragma unroll
                for (int t = KS - 2; t > 0; t--) win[t] = win[t - 1];
                win[0] = v;
                X[i + (size_t)ns * (j0 + c)] = v;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
typedef void (*chan_tridiag_fn)(int, int, const int *, const int *, const double *, const double *, double *,
                                double *, double *, double *, double *, double *, int *);
typedef void (*chan_back_fn)(int, int, int, const int *, const double *, const double *, const double *,
                             const double *, double *);

template <int KS> static void chan_fns(chan_tridiag_fn *t, chan_back_fn *b)
{
    *t = chan_tridiag_kernel<KS>;
    *b = chan_back_kernel<KS>;
}

static bool chan_lookup(int ks, chan_tridiag_fn *t, chan_back_fn *b)
{
    switch (ks) {
    case 2: chan_fns<2>(t, b); return true;
    case 3: chan_fns<3>(t, b); return true;
    case 4: chan_fns<4>(t, b); return true;
    case 5: chan_fns<5>(t, b); return true;
    case 6: chan_fns<6>(t, b); return true;
    case 7: chan_fns<7>(t, b); return true;
    case 8: chan_fns<8>(t, b); return true;
    case 9: chan_fns<9>(t, b); return true;
    case 10: chan_fns<10>(t, b); return true;
    case 11: chan_fns<11>(t, b); return true;
    case 12: chan_fns<12>(t, b); return true;
    case 13: chan_fns<13>(t, b); return true;
    case 14: chan_fns<14>(t, b); return true;
    case 15: chan_fns<15>(t, b); return true;
    case 16: chan_fns<16>(t, b); return true;
    default: return false;
    }
}

static size_t tridiag_smem(int npad, int ks) { return sizeof(double) * (tri(npad) + (size_t)npad * ks + 4 * (size_t)npad + 34); }

// panel width of the back-transform that fits the shared memory (0: none fits)
static int back_panel(int npad, int ks, size_t optin)
{
    const size_t fixed = tri(npad) + (size_t)npad + (size_t)npad * ks + 2 * (size_t)npad + CH_THREADS;
    for (int pw = 32; pw >= 8; pw /= 2) {
        const size_t bytes = sizeof(double) * (fixed + pw + (size_t)npad * (pw + 1));
        if (bytes <= optin) return pw;
    }
    return 0;
}

static size_t back_smem(int npad, int ks, int pw)
{
    return sizeof(double) * (tri(npad) + (size_t)npad + (size_t)npad * ks + 2 * (size_t)npad + pw + CH_THREADS +
                             (size_t)npad * (pw + 1));
}

bool chan_own_ok(int ns, int ks, int npad, int device)
{
    chan_tridiag_fn t;
    chan_back_fn b;
    if (!chan_lookup(ks, &t, &b) || npad > CH_NMAX || npad < 1) return false;
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    (void)ns;
    return tridiag_smem(npad, ks) <= (size_t)optin && back_panel(npad, ks, (size_t)optin) > 0;
}

size_t chan_own_workspace_doubles(int nch, int npad, int ks)
{
    const size_t np2 = (size_t)npad * npad;
    // X, Y, Y', G | L band | reflectors | d, e, tau | LU scratch (5 per channel)
    return (size_t)nch * (4 * np2 + (size_t)npad * ks + tri(npad) + 3 * (size_t)npad + 5 * np2) + 64;
}

int chan_own_solve(bsrg_ctx *c, const bsrg_basis *b, const double *hcc, int nch, int npad, const int *d_s0,
                   const int *d_nsol, double *AA, double *Wv, int *d_info, double *ws, int *d_flag)
{
    const int ns = b->ns, ks = b->ks;
    cudaStream_t s = c->stream;
    chan_tridiag_fn ktri;
    chan_back_fn kback;
    if (!chan_lookup(ks, &ktri, &kback)) { set_error("channel solves: ks=%d outside 2..16", ks); return BSRG_ERR_ARG; }
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
    const int pw = back_panel(npad, ks, (size_t)optin);
    const size_t sm1 = tridiag_smem(npad, ks), sm4 = back_smem(npad, ks, pw);
    if (pw == 0 || sm1 > (size_t)optin) { set_error("channel solves: n=%d too large for shared memory", npad); return BSRG_ERR_ARG; }
    const size_t np2 = (size_t)npad * npad;
    double *X = ws, *Y = X + np2 * nch, *Y2 = Y + np2 * nch, *Gm = Y2 + np2 * nch;
    double *Lg = Gm + np2 * nch, *Vg = Lg + (size_t)npad * ks * nch, *dg = Vg + tri(npad) * nch;
    double *eg = dg + (size_t)npad * nch, *tg = eg + (size_t)npad * nch, *scr = tg + (size_t)npad * nch;
    cudaError_t e;
    if ((e = smem_attr(ktri, (int)sm1)) != cudaSuccess ||
        (e = smem_attr(kback, (int)sm4)) != cudaSuccess)
        return cuda_fail(e, "channel solves: shared memory");
    if ((e = cudaMemsetAsync(d_flag, 0, 2 * sizeof(int), s)) != cudaSuccess) return cuda_fail(e, "channel solves: flag");
    ktri<<<nch, CH_THREADS, sm1, s>>>(ns, npad, d_s0, d_nsol, hcc, b->sb, X, Lg, Vg, dg, eg, tg, d_info);
    dim3 g2((unsigned)nch, (unsigned)((npad + 127) / 128));
    chan_eigvec_kernel<<<g2, 128, 0, s>>>(ns, npad, d_nsol, dg, eg, Wv, Y, scr);
    // two symmetric orthogonalisation steps; Y holds the eigenvectors as rows (Y^T column-major)
    double *src = Y, *dst = Y2;
    for (int pass = 0; pass < 2; pass++) {
        DgemmBatch g{};
        g.m = npad; g.n = npad; g.k = npad;
        g.A = src; g.lda = npad; g.sA = (long)np2;
        g.B = src; g.ldb = npad; g.sB = (long)np2;
        g.C = Gm; g.ldc = npad; g.sC = (long)np2;
        g.alpha = 1.0; g.beta = 0.0;
        int rc = dgemm_batched(false, true, g, nch, s);       // Gram matrix of the eigenvectors (rows)
        if (rc != BSRG_OK) return rc;
        dim3 gl((unsigned)((np2 + 255) / 256), (unsigned)nch);
        chan_lowdin_kernel<<<gl, 256, 0, s>>>(npad, d_nsol, Gm, pass == 0 ? d_flag : d_flag + 1);
        DgemmBatch u{};
        u.m = npad; u.n = npad; u.k = npad;
        u.A = Gm; u.lda = npad; u.sA = (long)np2;
        u.B = src; u.ldb = npad; u.sB = (long)np2;
        u.C = dst; u.ldc = npad; u.sC = (long)np2;
        u.alpha = 1.0; u.beta = 0.0;
        rc = dgemm_batched(false, false, u, nch, s);          // rows <- M rows
        if (rc != BSRG_OK) return rc;
        double *t = src; src = dst; dst = t;
    }
    kback<<<nch, CH_THREADS, sm4, s>>>(ns, npad, pw, d_nsol, Vg, tg, Lg, src, AA);
    return cuda_fail(cudaGetLastError(), "channel solves");
}

}  // namespace bsrg
