// density, convol and SUM_AmB of the reference's B-spline library on the GPU.
//
//   density (density.f90:2)  -> density_kernel
//   convol  (convol.f90:2)   -> direct_convol_kernel (icase 1,2), exchange_convol_kernel (icase 3,4)
//   SUM_AmB (sum_amb.f90:2)  -> sum_amb_kernel
//
// convol's exchange cases scatter each rkb element into up to four places of
// the result.  Here every output element gathers its contributions instead,
// which needs no atomics and is deterministic: with R(x,x',y,y') the R^k
// integral of the electron-1 pair (x,x') and electron-2 pair (y,y'),
//   icase 3:  a(x , y') = sum_{x',y} R(x,x',y,y') d(x',y)
//   icase 4:  a(x', y ) = sum_{x,y'} R(x,x',y,y') d(x,y')
// where R is read from rkb through the storage map of each electron: 's'
// (symmetric, rkb(min, ., |x-x'|+1, .)) or 'n' (rkb(x, ., x'-x+ks, .)).
// The direct cases (a band result) keep the reference's summation order with
// one thread per output element.  Compiled with --fmad=false.
#include "bsrg_internal.h"

namespace bsrg {

__global__ void density_kernel(int ns, int ks, double *d, const double *__restrict__ p1,
                               const double *__restrict__ p2, char type)
{
    int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (type == 's') {
        if (tid >= ns * ks) return;
        int i = tid % ns, j = tid / ns;
        double v = 0.0;
        if (j == 0) v = p1[i] * p2[i];
        else if (i < ns - j) v = p1[i] * p2[i + j] + p1[i + j] * p2[i];
        d[i + (size_t)ns * j] = v;
    } else if (type == 'n') {
        int k2 = 2 * ks - 1;
        if (tid >= ns * k2) return;
        int i = tid % ns, j = tid / ns;          // 0-based row, column (column j+1 in Fortran)
        int jj = i + j + 1 - ks;                 // partner index i + (j+1) - ks (0-based)
        double v = 0.0;
        if (jj >= 0 && jj < ns) v = p1[i] * p2[jj];
        d[i + (size_t)ns * j] = v;
    } else {
        if (tid >= ns * ns) return;
        int i = tid % ns, j = tid / ns;
        d[i + (size_t)ns * j] = p1[i] * p2[j];
    }
}

// band geometry: column c (0-based) of a band of storage 's' holds rows
// 0..ns-1-c; of storage 'n' holds rows max(0,ks-1-c)..min(ns-1, ns-1+ks-1-c)
__device__ __forceinline__ void band_rows(char sym, int ns, int ks, int c, int &lo, int &hi)
{
    if (sym == 's') { lo = 0; hi = ns - 1 - c; }
    else {
        lo = ks - 1 - c; if (lo < 0) lo = 0;
        hi = ns - 1 + ks - 1 - c; if (hi > ns - 1) hi = ns - 1;
    }
}

// icase 1: a(o,op) over band(sym_i) = sum over band(sym_j) (jp outer, j inner) d(j,jp) rkb(o,j,op,jp)
// icase 2: a(o,op) over band(sym_j) = sum over band(sym_i) (ip outer, i inner) d(i,ip) rkb(i,o,ip,op)
__global__ void direct_convol_kernel(int ns, int ks, int ldp, int icase, char si, char sj, double *a,
                                     const double *__restrict__ d, const double *__restrict__ rkb)
{
    char so = icase == 1 ? si : sj;    // output band storage
    char sc = icase == 1 ? sj : si;    // contracted band storage
    int nco = so == 's' ? ks : 2 * ks - 1;
    int ncc = sc == 's' ? ks : 2 * ks - 1;
    int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= ns * nco) return;
    int o = tid % ns, op = tid / ns;
    int lo, hi;
    band_rows(so, ns, ks, op, lo, hi);
    if (o < lo || o > hi) return;       // the reference leaves those entries untouched
    size_t nn = (size_t)ns * ns;
    double c = 0.0;
    for (int cp = 0; cp < ncc; cp++) {
        int clo, chi;
        band_rows(sc, ns, ks, cp, clo, chi);
        for (int q = clo; q <= chi; q++) {
            size_t r = icase == 1 ? (o + (size_t)ns * q + nn * (op + (size_t)ldp * cp))
                                  : (q + (size_t)ns * o + nn * (cp + (size_t)ldp * op));
            c = c + d[q + (size_t)ns * cp] * rkb[r];
        }
    }
    a[o + (size_t)ns * op] = c;
}

// map an electron pair (x, x') to (stored row, stored column index) of rkb;
// returns false if the pair has no entry.
__device__ __forceinline__ bool pair_map(char sym, int ns, int ks, int x, int xp, int &row, int &col)
{
    int dx = xp - x;
    if (dx <= -ks || dx >= ks || x < 0 || xp < 0 || x >= ns || xp >= ns) return false;
    if (sym == 's') { row = dx >= 0 ? x : xp; col = dx >= 0 ? dx : -dx; }
    else { row = x; col = dx + ks - 1; }
    return true;
}

__global__ void exchange_convol_kernel(int ns, int ks, int ldp, int icase, char si, char sj, double *a,
                                       const double *__restrict__ d, const double *__restrict__ rkb)
{
    int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= ns * ns) return;
    int u = tid % ns, v = tid / ns;     // output a(u, v)
    size_t nn = (size_t)ns * ns;
    double c = 0.0;
    for (int e = -(ks - 1); e <= ks - 1; e++) {
        for (int f = -(ks - 1); f <= ks - 1; f++) {
            int x, xp, y, yp;
            if (icase == 3) { x = u; xp = u + e; yp = v; y = v + f; }   // a(x,y') <- d(x',y)
            else { xp = u; x = u + e; y = v; yp = v + f; }              // a(x',y) <- d(x,y')
            int r1, c1, r2, c2;
            if (!pair_map(si, ns, ks, x, xp, r1, c1)) continue;
            if (!pair_map(sj, ns, ks, y, yp, r2, c2)) continue;
            double rv = rkb[r1 + (size_t)ns * r2 + nn * (c1 + (size_t)ldp * c2)];
            double dv = icase == 3 ? d[xp + (size_t)ns * y] : d[x + (size_t)ns * yp];
            c = c + rv * dv;
        }
    }
    a[u + (size_t)ns * v] = c;
}

__global__ void sum_amb_kernel(int ns, int ks, const double *a, const double *b, char sym, double *out)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    double x = 0.0;
    if (sym == 'x') {
        for (int i = 0; i < ns; i++)
            for (int j = 0; j < ns; j++) x = x + a[i + (size_t)ns * j] * b[i + (size_t)ns * j];
    } else if (sym == 's') {
        for (int j = 1; j <= ks; j++)
            for (int i = 1; i <= ns - j + 1; i++)
                x = x + a[(i - 1) + (size_t)ns * (j - 1)] * b[(i - 1) + (size_t)ns * (j - 1)];
    } else if (sym == 'l') {
        for (int j = 1; j <= ks; j++)
            for (int i = ks + 1 - j; i <= ns; i++)
                x = x + a[(i - 1) + (size_t)ns * (j - 1)] * b[(i - 1) + (size_t)ns * (j - 1)];
    } else {
        for (int j = 1; j <= 2 * ks - 1; j++) {
            int imin = 1 > 1 + ks - j ? 1 : 1 + ks - j;
            int imax = ns < ns + ks - j ? ns : ns + ks - j;
            for (int i = imin; i <= imax; i++)
                x = x + a[(i - 1) + (size_t)ns * (j - 1)] * b[(i - 1) + (size_t)ns * (j - 1)];
        }
    }
    *out = x;
}

int launch_density(int ns, int ks, double *d, const double *p1, const double *p2, char type, cudaStream_t s)
{
    int n = type == 's' ? ns * ks : (type == 'n' ? ns * (2 * ks - 1) : ns * ns);
    density_kernel<<<(n + 127) / 128, 128, 0, s>>>(ns, ks, d, p1, p2, type);
    return cuda_fail(cudaGetLastError(), "density");
}

int launch_convol(int ns, int ks, double *a, const double *d, const double *rkb, int ldp, int icase, char si,
                  char sj, cudaStream_t s)
{
    if (icase == 1 || icase == 2) {
        char so = icase == 1 ? si : sj;
        int n = ns * (so == 's' ? ks : 2 * ks - 1);
        direct_convol_kernel<<<(n + 127) / 128, 128, 0, s>>>(ns, ks, ldp, icase, si, sj, a, d, rkb);
    } else {
        int n = ns * ns;
        exchange_convol_kernel<<<(n + 127) / 128, 128, 0, s>>>(ns, ks, ldp, icase, si, sj, a, d, rkb);
    }
    return cuda_fail(cudaGetLastError(), "convol");
}

int launch_sum_amb(int ns, int ks, const double *a, const double *b, char sym, double *out, cudaStream_t s)
{
    sum_amb_kernel<<<1, 32, 0, s>>>(ns, ks, a, b, sym, out);
    return cuda_fail(cudaGetLastError(), "sum_amb");
}

// bav (bav.f90:2): y = B v ('s'; 'n' with side 'r') or y = v B ('n', side 'l').  One thread
// per output, the terms added in the order the reference's scatter loops reach that output
// (for 's': within each diagonal ip the transposed term b(x-ip+1, ip) v(x-ip+1) comes first).
__global__ void bav_kernel(int ns, int ks, const double *__restrict__ b, const double *__restrict__ v, double *y,
                           char type, char side)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;   // 0-based output index
    if (x >= ns) return;
    double acc;
    if (type == 's') {
        acc = b[x] * v[x];
        for (int ip = 2; ip <= ks; ip++) {
            const int i1 = x - ip + 1;            // row i whose j = i + ip - 1 is x
            if (i1 >= 0) acc = acc + b[i1 + (size_t)ns * (ip - 1)] * v[i1];
            if (x <= ns - ip) acc = acc + b[x + (size_t)ns * (ip - 1)] * v[x + ip - 1];
        }
    } else {
        acc = 0.0;
        for (int ip = 1; ip <= ks + ks - 1; ip++) {
            const int imin = max(1, 1 + ks - ip), imax = min(ns, ns + ks - ip);
            if (side == 'r') {
                const int i = x + 1, j = i + ip - ks;
                if (i >= imin && i <= imax) acc = acc + b[(i - 1) + (size_t)ns * (ip - 1)] * v[j - 1];
            } else {
                const int i = x + 1 - ip + ks;     // j = i + ip - ks = x + 1
                if (i >= imin && i <= imax) acc = acc + b[(i - 1) + (size_t)ns * (ip - 1)] * v[i - 1];
            }
        }
    }
    y[x] = acc;
}

// bvmv (bvmv.f90:2): <x, A y> for a band array, in the reference's summation order
// (one thread: the sum is a single ordered accumulation of O(n k) terms)
__device__ double bvmv_dev(int n, int k, const double *ar, char type, const double *x, const double *y)
{
    double s = 0.0;
    if (type != 'g') {
        for (int jp = 1; jp <= k - 1; jp++)
            for (int i = k + 1 - jp; i <= n; i++) {
                const int j = i + jp - k;
                s = s + ar[(i - 1) + (size_t)n * (jp - 1)] * (x[i - 1] * y[j - 1] + x[j - 1] * y[i - 1]);
            }
        if (type == 'a') s = s + x[n - 2] * y[n - 1] * (ar[0] - ar[(n - 1) + (size_t)n * (k - 2)]);
    } else {
        for (int jp = 1; jp <= k - 1; jp++)
            for (int i = k - jp + 1; i <= n; i++) {
                const int j = i + jp - k, kp = 2 * k - jp;
                s = s + ar[(i - 1) + (size_t)n * (jp - 1)] * x[i - 1] * y[j - 1];
                s = s + ar[(j - 1) + (size_t)n * (kp - 1)] * x[j - 1] * y[i - 1];
            }
    }
    double c = 0.0;
    for (int i = 1; i <= n; i++) c = c + ar[(i - 1) + (size_t)n * (k - 1)] * x[i - 1] * y[i - 1];
    return s + c;
}

__global__ void bvmv_kernel(int n, int k, const double *ar, char type, const double *x, const double *y, double *out)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) *out = bvmv_dev(n, k, ar, type, x, y);
}

int launch_bav(int ns, int ks, const double *b, const double *v, double *y, char type, char side, cudaStream_t s)
{
    bav_kernel<<<(ns + 127) / 128, 128, 0, s>>>(ns, ks, b, v, y, type, side);
    return cuda_fail(cudaGetLastError(), "bav");
}

int launch_bvmv(int n, int k, const double *ar, char type, const double *x, const double *y, double *out,
                cudaStream_t s)
{
    bvmv_kernel<<<1, 32, 0, s>>>(n, k, ar, type, x, y, out);
    return cuda_fail(cudaGetLastError(), "bvmv");
}

}  // namespace bsrg
