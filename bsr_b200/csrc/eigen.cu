// Dense symmetric eigensolver pieces for sm_100a: Householder tridiagonal reduction.
//
// DSYEV (called by diag_hd through LAP_DSYEV, ZCOM/LAPACK_calls.f90:54-76) spends
// its time in the reduction A = Q T Q^T.  The one-stage blocked reduction
// (LAPACK dsytrd/dlatrd, uplo = 'L') is kept, but each panel of TRD_NB columns
// runs as ONE cooperative kernel: per column a row-parallel update of the
// column, a grid barrier, the reflector, the symmetric matrix-vector product
// with the trailing matrix (tiles of the lower triangle, each read once) plus
// the panel corrections, and a second grid barrier.  The rank-2k trailing
// update between panels is cuBLAS DSYR2K.  Every cross-CTA sum is written to
// its own slot and added in a fixed order, so results are bitwise repeatable.
//
// Output follows LAPACK dsytrd lower: d, e, tau, and the reflector vectors in
// A below the subdiagonal (v(c+1) = 1 implicit), so DORMTR applies Q.
#include <cuda_runtime.h>

#include <cmath>

#include "ctx.h"

namespace bsrg {
namespace {

constexpr int TRD_NB = 32;                  // panel width
constexpr int TRD_TT = 64;                  // tile edge of the symmetric product
constexpr int TRD_BB = 4;                   // largest tiles per block edge (a work unit is one block)
constexpr int TRD_BT = TRD_TT * TRD_BB;     // largest block edge
constexpr int TRD_NT = 512;                 // threads per CTA
constexpr int TRD_CG = TRD_NT / TRD_TT;     // column groups in a tile
constexpr int TRD_CPT = TRD_TT / TRD_CG;    // columns per thread in a tile
constexpr int TRD_G = 8;                    // lanes per row in the row phase
constexpr int TRD_RPC = TRD_NT / TRD_G;     // rows per CTA pass in the row phase
constexpr int TRD_DR = 256;                 // rows per dot chunk
constexpr int TRD_LDT = TRD_TT + 1;         // padded leading dimension of a staged tile
constexpr int TRD_SMEM = (2 * TRD_TT * TRD_LDT + TRD_CG * TRD_BT + 2 * TRD_BT) * 8;   // dynamic shared bytes
constexpr long TRD_SPIN_LIMIT = 1L << 24;   // barrier spin bound (an error, never expected)

struct TrdArgs {
    double *A;
    int n, lda;
    int p0, nbp;            // first column of the panel, columns in the panel
    double *W;              // n x TRD_NB (ld n): w vectors of the panel
    double *d, *e, *tau;
    double *P;              // nblk x n: row partials of the product, by block column
    double *Q;              // nblk x n: column partials, by block row
    double *col;            // n: the current column after its update
    double *red_norm;       // per CTA
    double *red_dot;        // per dot chunk: 2*TRD_NB
    double *red_s1;         // per CTA
    unsigned *bar;          // [2] dynamic work counter
    unsigned *arrive;       // per CTA (stride 8): last barrier generation reached
    unsigned *release;      // generation released by CTA 0
    int *err;
    unsigned gen0;          // barrier generations of this launch start above gen0
};

// Grid barrier: every CTA publishes the generation it reached in its own slot;
// CTA 0 waits for all slots, resets the work counter and publishes the release.
// Every wait is bounded; on a timeout the error flag ends the kernel.
__device__ __forceinline__ bool grid_barrier(const TrdArgs &a, unsigned gen)
{
    __syncthreads();
    const int t = threadIdx.x, cta = blockIdx.x;
    volatile int *verr = a.err;
    if (t == 0) {
        __threadfence();
        *(volatile unsigned *)(a.arrive + 8 * cta) = gen;
    }
    if (cta == 0) {
        if (t < (int)gridDim.x) {
            long it = 0;
            while (*(volatile unsigned *)(a.arrive + 8 * t) != gen && *verr == 0)
                if (++it > TRD_SPIN_LIMIT) atomicExch(a.err, 1);
        }
        __syncthreads();
        if (t == 0) {
            __threadfence();
            *(volatile unsigned *)(a.bar + 2) = 0u;
            __threadfence();
            *(volatile unsigned *)a.release = gen;
        }
    } else if (t == 0) {
        long it = 0;
        while (*(volatile unsigned *)a.release != gen && *verr == 0)
            if (++it > TRD_SPIN_LIMIT) atomicExch(a.err, 1);
    }
    if (t == 0) __threadfence();
    __syncthreads();
    return *verr == 0;
}

// tiles per block edge for a trailing matrix of m rows: the largest that still
// gives every CTA two work units (small m: 64 x 64 units, large m: 256 x 256)
__host__ __device__ __forceinline__ int bb_for(int m, int ncta)
{
    for (int bb = TRD_BB; bb > 1; bb >>= 1) {
        const int nb = (m + TRD_TT * bb - 1) / (TRD_TT * bb);
        if (nb * (nb + 1) / 2 >= 2 * ncta) return bb;
    }
    return 1;
}

__device__ __forceinline__ double vval(const double *col, int r, int c, int n, double scale)
{
    if (r <= c || r >= n) return 0.0;
    return r == c + 1 ? 1.0 : col[r] * scale;
}

// block sum of one value per thread, fixed order; result valid in every thread
__device__ double block_sum(double v, double *sh)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double s = 0.0;
    for (int w = 0; w < TRD_NT / 32; w++) s += sh[w];
    __syncthreads();
    return s;
}

// Row phase for row r (8 lanes; every lane of the warp calls it, act = row exists):
// py = y_r of the product of column c-1 (its blocks of bt rows), pc = the panel
// corrections of that product (l < i-1), pu = the update of column c at row r by
// panel columns l < i-1.  The l = i-1 terms need W(c, i-1), added by the caller.
struct RowSums {
    double py, pc, pu;
};

__device__ __forceinline__ RowSums row_sums(const TrdArgs &a, int r, bool act, int c, int i, int bt,
                                            const double *sxw, const double *sxv, const double *sWc,
                                            const double *sVc)
{
    const int lane = threadIdx.x & (TRD_G - 1);
    const int n = a.n, lda = a.lda;
    double py0 = 0.0, py1 = 0.0, pc = 0.0, pu = 0.0;
    if (act) {
        if (i > 0) {
            const int IBr = r / bt;
            const int JB0 = c / bt;                   // blocks of the product of column c-1
            const int nblk = (n + bt - 1) / bt;
#pragma unroll 4
            for (int JB = JB0 + lane; JB <= IBr; JB += TRD_G) py0 += a.P[(size_t)JB * n + r];
#pragma unroll 4
            for (int IB = IBr + lane; IB < nblk; IB += TRD_G) py1 += a.Q[(size_t)IB * n + r];
        }
#pragma unroll 4
        for (int l = lane; l < i - 1; l += TRD_G) {
            const double v = a.A[r + (size_t)(a.p0 + l) * lda];
            const double w = a.W[r + (size_t)l * n];
            pc += v * sxw[l] + w * sxv[l];
            pu += v * sWc[l] + w * sVc[l];
        }
    }
    double py = py0 + py1;
#pragma unroll
    for (int o = TRD_G / 2; o > 0; o >>= 1) {
        py += __shfl_xor_sync(0xffffffffu, py, o);
        pc += __shfl_xor_sync(0xffffffffu, pc, o);
        pu += __shfl_xor_sync(0xffffffffu, pu, o);
    }
    return {py, pc, pu};
}

// one block (IB, JB) of bb x bb tiles of y = A22 v, JB <= IB: the 64 x 64
// tiles of the lower triangle are staged through shared memory
// (double-buffered, two tiles of loads in flight) and each is read once; row
// sums go to P(JB, rows), transposed sums to Q(IB, cols); s1acc collects
// v^T (A22 v) of what it writes.
__device__ void product_unit(const TrdArgs &a, int c, double scale, int IB, int JB, int bb, double *smem,
                             double &s1acc)
{
    const int n = a.n, lda = a.lda, t = threadIdx.x;
    const int tr = t % TRD_TT, g = t / TRD_TT;
    const int bt = bb * TRD_TT;
    const double *A = a.A;
    double *tile0 = smem, *tile1 = smem + TRD_TT * TRD_LDT;
    double *red = smem + 2 * TRD_TT * TRD_LDT;                 // TRD_CG x TRD_BT
    double *vI = red + TRD_CG * TRD_BT, *vJ = vI + TRD_BT;
    const bool diag = (IB == JB);
    const int ntile = diag ? bb * (bb + 1) / 2 : bb * bb;
    auto tile_of = [&](int q, int &il, int &jl) {
        if (!diag) {
            il = q / bb;
            jl = q % bb;
        } else {
            il = 0;
            while (q > il) {
                q -= il + 1;
                il++;
            }
            jl = q;
        }
    };
    auto load = [&](int q, double *dst) {
        int il, jl;
        tile_of(q, il, jl);
        const int I = IB * bb + il, J = JB * bb + jl;
        const int r = I * TRD_TT + tr;
#pragma unroll
        for (int k = 0; k < TRD_CPT; k++) {
            const int sc = J * TRD_TT + g + k * TRD_CG;
            const bool ok = r < n && sc < n && (I > J || r >= sc);
            dst[k] = ok ? A[r + (size_t)sc * lda] : 0.0;
        }
    };
    double ra[TRD_CPT], rb[TRD_CPT];
    load(0, ra);
    if (ntile > 1) load(1, rb);
    if (t < bt) {
        vI[t] = vval(a.col, IB * bt + t, c, n, scale);
        vJ[t] = vval(a.col, JB * bt + t, c, n, scale);
    }
    double rowacc[TRD_BB], zacc[TRD_BB];
#pragma unroll
    for (int q = 0; q < TRD_BB; q++) rowacc[q] = zacc[q] = 0.0;
    for (int q = 0; q < ntile; q++) {
        double *T = (q & 1) ? tile1 : tile0;
#pragma unroll
        for (int k = 0; k < TRD_CPT; k++) T[(g + k * TRD_CG) * TRD_LDT + tr] = ra[k];
#pragma unroll
        for (int k = 0; k < TRD_CPT; k++) ra[k] = rb[k];
        if (q + 2 < ntile) load(q + 2, rb);
        __syncthreads();
        int il, jl;
        tile_of(q, il, jl);
        const bool dtile = diag && il == jl;
        {
            double sacc = 0.0;
#pragma unroll
            for (int k = 0; k < TRD_CPT; k++) {
                const int sl = g * TRD_CPT + k;
                sacc += T[sl * TRD_LDT + tr] * vJ[jl * TRD_TT + sl];
            }
#pragma unroll
            for (int qq = 0; qq < TRD_BB; qq++)
                if (qq == il) rowacc[qq] += sacc;
        }
        {
            double sacc = 0.0;
#pragma unroll
            for (int k = 0; k < TRD_CPT; k++) {
                const int rl = g * TRD_CPT + k;
                const double x = T[tr * TRD_LDT + rl] * vI[il * TRD_TT + rl];
                sacc += (!dtile || rl > tr) ? x : 0.0;
            }
#pragma unroll
            for (int qq = 0; qq < TRD_BB; qq++)
                if (qq == jl) zacc[qq] += sacc;
        }
    }
#pragma unroll
    for (int q = 0; q < TRD_BB; q++)
        if (q < bb) red[g * TRD_BT + q * TRD_TT + tr] = rowacc[q];
    __syncthreads();
    if (t < bt) {
        double y = 0.0;
#pragma unroll
        for (int gg = 0; gg < TRD_CG; gg++) y += red[gg * TRD_BT + t];
        const int rr = IB * bt + t;
        if (rr < n) {
            a.P[(size_t)JB * n + rr] = y;
            s1acc += vI[t] * y;
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < TRD_BB; q++)
        if (q < bb) red[g * TRD_BT + q * TRD_TT + tr] = zacc[q];
    __syncthreads();
    if (t < bt) {
        double z = 0.0;
#pragma unroll
        for (int gg = 0; gg < TRD_CG; gg++) z += red[gg * TRD_BT + t];
        const int cc = JB * bt + t;
        if (cc < n) {
            a.Q[(size_t)IB * n + cc] = z;
            s1acc += vJ[t] * z;
        }
    }
    __syncthreads();
}

// V^T v and W^T v over one chunk of TRD_DR rows (previous panel columns l < i)
__device__ void dot_chunk(const TrdArgs &a, int c, double scale, int i, int dq, double *sh)
{
    const int n = a.n, t = threadIdx.x;
    const int tr = t % TRD_TT, cg = t / TRD_TT;
    constexpr int NQ = TRD_NB / TRD_CG;
    double pw[NQ], pv[NQ];
#pragma unroll
    for (int q = 0; q < NQ; q++) pw[q] = pv[q] = 0.0;
#pragma unroll
    for (int rk = 0; rk < TRD_DR / TRD_TT; rk++) {
        const int r = c + 1 + dq * TRD_DR + rk * TRD_TT + tr;
        const double vr = vval(a.col, r, c, n, scale);
#pragma unroll
        for (int q = 0; q < NQ; q++) {
            const int l = cg + q * TRD_CG;
            if (l < i && r < n) {
                pw[q] += a.W[r + (size_t)l * n] * vr;
                pv[q] += a.A[r + (size_t)(a.p0 + l) * a.lda] * vr;
            }
        }
    }
#pragma unroll
    for (int q = 0; q < NQ; q++) {
        for (int o = 16; o > 0; o >>= 1) {
            pw[q] += __shfl_xor_sync(0xffffffffu, pw[q], o);
            pv[q] += __shfl_xor_sync(0xffffffffu, pv[q], o);
        }
    }
    const int lane = t & 31, half = tr / 32;
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < NQ; q++) {
            sh[(cg * NQ + q) * 2 + half] = pw[q];
            sh[TRD_NB * 2 + (cg * NQ + q) * 2 + half] = pv[q];
        }
    }
    __syncthreads();
    if (t < TRD_NB) {
        const int l = t, idx = (l % TRD_CG) * NQ + l / TRD_CG;
        a.red_dot[(size_t)dq * 2 * TRD_NB + l] = sh[idx * 2] + sh[idx * 2 + 1];
        a.red_dot[(size_t)dq * 2 * TRD_NB + TRD_NB + l] = sh[TRD_NB * 2 + idx * 2] + sh[TRD_NB * 2 + idx * 2 + 1];
    }
    __syncthreads();
}

constexpr int TRD_MAXPASS = 4;              // row passes per CTA: n <= 4 * 64 * (number of CTAs)

__global__ void __launch_bounds__(TRD_NT, 1) trd_panel_kernel(TrdArgs a)
{
    extern __shared__ double dsm[];             // staged tiles and block reductions (TRD_SMEM bytes)
    double *sh = dsm;                           // also the scratch of the small reductions
    __shared__ int snext;
    __shared__ double sxw[TRD_NB], sxv[TRD_NB], sWc[TRD_NB], sVc[TRD_NB];
    __shared__ double sbc[4];
    const int t = threadIdx.x, cta = blockIdx.x, ncta = gridDim.x;
    const int n = a.n, lda = a.lda;
    double *A = a.A;
    unsigned gen = a.gen0;
    double tau_p = 0.0, alpha2_p = 0.0;          // of the previous column (same in every CTA)
    int bt_p = TRD_TT;                          // block edge of the previous column's product
    for (int i = 0; i <= a.nbp; i++) {
        // column c = p0 + i; i == nbp only finishes w of the last panel column
        // (and the last diagonal element when c == n-1)
        const int c = a.p0 + i;
        const bool last = (i == a.nbp);
        // ---- row phase: finish w of column c-1 at rows >= c, update column c ----
        // sVc(0:i-1) and sWc(0:i-2) hold row c of V and W (loaded after the last barrier)
        RowSums rs[TRD_MAXPASS];
        double vr[TRD_MAXPASS], arc[TRD_MAXPASS];
#pragma unroll
        for (int q = 0; q < TRD_MAXPASS; q++) {
            const int base = c + (cta + q * ncta) * TRD_RPC;     // the same in the whole CTA
            rs[q] = {0.0, 0.0, 0.0};
            vr[q] = arc[q] = 0.0;
            if (base < n) {
                const int r = base + t / TRD_G;
                const bool act = r < n;
                rs[q] = row_sums(a, r, act, c, i, bt_p, sxw, sxv, sWc, sVc);
                vr[q] = (act && i > 0) ? A[r + (size_t)(c - 1) * lda] : 0.0;
                arc[q] = act ? A[r + (size_t)c * lda] : 0.0;
            }
        }
        if (i > 0 && t < 32) {
            // W(c, i-1), needed by every row: every CTA computes it with the row code
            const RowSums rc = row_sums(a, c, t < TRD_G, c, i, bt_p, sxw, sxv, sWc, sVc);
            if (t == 0) sWc[i - 1] = tau_p * (rc.py - rc.pc) + alpha2_p * A[c + (size_t)(c - 1) * lda];
        }
        __syncthreads();
        double nrm = 0.0;
#pragma unroll
        for (int q = 0; q < TRD_MAXPASS; q++) {
            const int r = c + (cta + q * ncta) * TRD_RPC + t / TRD_G;
            if (r < n && (t & (TRD_G - 1)) == 0) {
                double wr = 0.0, ar = arc[q] - rs[q].pu;
                if (i > 0) {
                    wr = tau_p * (rs[q].py - rs[q].pc) + alpha2_p * vr[q];
                    a.W[r + (size_t)(i - 1) * n] = wr;
                    ar -= vr[q] * sWc[i - 1] + wr * sVc[i - 1];
                }
                if (!last || c == n - 1) {
                    a.col[r] = ar;
                    if (r == c) {
                        a.d[c] = ar;
                        A[c + (size_t)c * lda] = ar;
                    }
                    if (r >= c + 2) nrm += ar * ar;
                }
            }
        }
        if (last) break;
        nrm = block_sum(nrm, sh);
        if (t == 0) a.red_norm[cta] = nrm;
        if (!grid_barrier(a, ++gen)) return;
        // ---- reflector, product, dots ----
        const int m = n - c;
        {
            double sq = (t < ncta) ? a.red_norm[t] : 0.0;
            const double alpha = a.col[c + 1];
            sq = block_sum(sq, sh);
            if (t == 0) {
                double beta, tau, scale;
                if (sq == 0.0) {
                    beta = alpha;
                    tau = 0.0;
                    scale = 0.0;
                } else {
                    beta = -copysign(sqrt(alpha * alpha + sq), alpha);
                    tau = (beta - alpha) / beta;
                    scale = 1.0 / (alpha - beta);
                }
                sbc[1] = beta;
                sbc[2] = tau;
                sbc[3] = scale;
            }
            __syncthreads();
        }
        const double tau = sbc[2], scale = sbc[3];
        if (cta == 0 && t == 0) {
            a.e[c] = sbc[1];
            a.tau[c] = tau;
        }
        for (int q = cta; q * TRD_NT < m - 1; q += ncta) {
            const int r = c + 1 + q * TRD_NT + t;
            if (r < n) A[r + (size_t)c * lda] = vval(a.col, r, c, n, scale);
        }
        const int bb = bb_for(m - 1, ncta);
        const int bt = bb * TRD_TT;
        const int nblk = (n + bt - 1) / bt;
        const int jb0 = (c + 1) / bt;
        const int nb = nblk - jb0;
        const int noff = nb * (nb - 1) / 2;        // off-diagonal blocks first (largest), then diagonal ones
        const int nunit = noff + nb;
        const int ndot = (i > 0) ? (m - 1 + TRD_DR - 1) / TRD_DR : 0;
        double s1acc = 0.0;
        int u = cta;
        while (u < nunit + ndot) {
            if (t == 0) snext = (int)atomicAdd(a.bar + 2, 1u) + ncta;   // next unit, fetched ahead
            if (u < noff) {
                int uu = u, JB = jb0;
                while (uu >= nblk - JB - 1) {
                    uu -= nblk - JB - 1;
                    JB++;
                }
                product_unit(a, c, scale, JB + 1 + uu, JB, bb, dsm, s1acc);
            } else if (u < nunit) {
                const int JB = jb0 + (u - noff);
                product_unit(a, c, scale, JB, JB, bb, dsm, s1acc);
            } else {
                dot_chunk(a, c, scale, i, u - nunit, sh);
            }
            __syncthreads();
            u = snext;
            __syncthreads();
        }
        s1acc = block_sum(s1acc, sh);
        if (t == 0) a.red_s1[cta] = s1acc;
        if (!grid_barrier(a, ++gen)) return;
        // ---- every CTA: sums of the dots and of v^T A22 v, alpha2; rows c+1 of V and W ----
        {
            const int l = t % (2 * TRD_NB), g = t / (2 * TRD_NB);
            double sd = 0.0;
            for (int dq = g; dq < ndot; dq += TRD_NT / (2 * TRD_NB)) sd += a.red_dot[(size_t)dq * 2 * TRD_NB + l];
            const double s1p = (t < ncta) ? a.red_s1[t] : 0.0;
            // next column's row of V (l <= i) and W (l < i; W(c+1, i) comes from the row phase)
            double vnext = 0.0, wnext = 0.0;
            if (t <= i) vnext = A[c + 1 + (size_t)(a.p0 + t) * lda];
            if (t < i) wnext = a.W[c + 1 + (size_t)t * n];
            sh[g * 2 * TRD_NB + l] = sd;
            __syncthreads();
            if (t < 2 * TRD_NB) {
                double tot = 0.0;
                for (int gg = 0; gg < TRD_NT / (2 * TRD_NB); gg++) tot += sh[gg * 2 * TRD_NB + t];
                if (t < TRD_NB) sxw[t] = (t < i) ? tot : 0.0;
                else sxv[t - TRD_NB] = (t - TRD_NB < i) ? tot : 0.0;
            }
            const double s1 = block_sum(s1p, sh);    // its leading barrier orders the sxw/sxv writes
            double xx = 0.0;
            for (int ll = 0; ll < i; ll++) xx += sxv[ll] * sxw[ll];
            const double wv = s1 - 2.0 * xx;
            tau_p = tau;
            alpha2_p = -0.5 * tau * tau * wv;
            bt_p = bt;
            if (t <= i) sVc[t] = vnext;
            if (t < i) sWc[t] = wnext;
            __syncthreads();
        }
    }
}

__global__ void trd_restore_e_kernel(int n, double *A, int lda, const double *e)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < n - 1) A[c + 1 + (size_t)c * lda] = e[c];
}

}  // namespace

// workspace layout of one reduction (the same carve for the launch and the error check)
struct TrdLayout {
    double *W, *P, *Q, *col, *red_norm, *red_dot, *red_s1;
    unsigned *bar, *arrive, *release;
    int *err;
    size_t bytes;
};

static TrdLayout trd_layout(void *ws, int n)
{
    const size_t nt = (n + TRD_TT - 1) / TRD_TT;       // partial rows for the smallest blocks
    const size_t ndot = (n + TRD_DR - 1) / TRD_DR;
    Arena ar{(char *)ws, 0, 0};
    TrdLayout L{};
    L.W = ar.take<double>((size_t)n * TRD_NB);
    L.P = ar.take<double>(nt * n);
    L.Q = ar.take<double>(nt * n);
    L.col = ar.take<double>(n);
    L.red_norm = ar.take<double>(TRD_NT);
    L.red_dot = ar.take<double>(ndot * 2 * TRD_NB);
    L.red_s1 = ar.take<double>(TRD_NT);
    L.bar = ar.take<unsigned>(16);                      // [2] work counter, [8] error flag
    L.err = (int *)(L.bar + 8);
    L.arrive = ar.take<unsigned>(8 * TRD_NT);
    L.release = ar.take<unsigned>(16);
    L.bytes = ar.off + 256;
    return L;
}

size_t trd_workspace_bytes(int n) { return trd_layout(nullptr, n).bytes; }

// A (n x n, lower triangle) -> T (d, e) and reflectors; ws holds trd_workspace_bytes(n)
int trd_reduce(bsrg_ctx *c, int n, double *A, int lda, double *d, double *e, double *tau, void *ws)
{
    cudaStream_t s = c->stream;
    if (n < 1) return BSRG_OK;
    if (n == 1) {
        cudaError_t er = cudaMemcpyAsync(d, A, sizeof(double), cudaMemcpyDeviceToDevice, s);
        return er == cudaSuccess ? BSRG_OK : cuda_fail(er, "tridiagonal reduction");
    }
    const TrdLayout L = trd_layout(ws, n);
    TrdArgs a{};
    a.A = A;
    a.n = n;
    a.lda = lda;
    a.W = L.W;
    a.P = L.P;
    a.Q = L.Q;
    a.col = L.col;
    a.red_norm = L.red_norm;
    a.red_dot = L.red_dot;
    a.red_s1 = L.red_s1;
    a.bar = L.bar;
    a.err = L.err;
    a.arrive = L.arrive;
    a.release = L.release;
    a.d = d;
    a.e = e;
    a.tau = tau;
    cudaError_t er;
    // flags start at generation 0; every launch uses generations above its own gen0
    const size_t flag_bytes = (char *)(L.release + 16) - (char *)L.bar;
    if ((er = cudaMemsetAsync(L.bar, 0, flag_bytes, s)) != cudaSuccess) return cuda_fail(er, "tridiagonal reduction");
    int dev = c->device, nsm = 0, occ = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if ((er = smem_attr(trd_panel_kernel, TRD_SMEM)) !=
        cudaSuccess)
        return cuda_fail(er, "tridiagonal reduction smem");
    if ((er = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, trd_panel_kernel, TRD_NT, TRD_SMEM)) != cudaSuccess)
        return cuda_fail(er, "tridiagonal reduction occupancy");
    if (occ < 1) {
        set_error("tridiagonal reduction: kernel cannot be resident");
        return BSRG_ERR_CUDA;
    }
    // one CTA per SM, all resident (the cooperative launch checks it); the
    // per-CTA slots are read by one thread each, so at most TRD_NT CTAs
    const int grid = nsm < TRD_NT ? nsm : TRD_NT;
    if (n > TRD_MAXPASS * TRD_RPC * grid) {
        set_error("tridiagonal reduction: n = %d above the limit %d of this device", n, TRD_MAXPASS * TRD_RPC * grid);
        return BSRG_ERR_ARG;
    }
    const double one = 1.0, mone = -1.0;
    unsigned launch = 0;
    for (int p0 = 0; p0 < n - 1; p0 += TRD_NB) {
        a.p0 = p0;
        a.nbp = min(TRD_NB, n - 1 - p0);
        a.gen0 = ++launch * 256u;            // at most 2 * TRD_NB barriers per launch
        void *args[] = {&a};
        if ((er = cudaLaunchCooperativeKernel((const void *)trd_panel_kernel, grid, TRD_NT, args, TRD_SMEM, s)) !=
            cudaSuccess)
            return cuda_fail(er, "tridiagonal reduction panel");
        const int q0 = p0 + a.nbp;
        if (q0 < n - 1) {
            const int mm = n - q0;
            cublasStatus_t bs = cublasDsyr2k(c->blas, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, mm, a.nbp, &mone,
                                             A + q0 + (size_t)p0 * lda, lda, a.W + q0, n, &one,
                                             A + q0 + (size_t)q0 * lda, lda);
            if (bs != CUBLAS_STATUS_SUCCESS) {
                set_error("tridiagonal reduction: DSYR2K failed (%d)", (int)bs);
                return BSRG_ERR_SOLVER;
            }
        }
    }
    trd_restore_e_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, A, lda, e);
    if ((er = cudaGetLastError()) != cudaSuccess) return cuda_fail(er, "tridiagonal reduction");
    return BSRG_OK;
}

// error flag of the last reduction (read after the stream is synchronised)
int trd_check(void *ws, int n, cudaStream_t s)
{
    const TrdLayout L = trd_layout(ws, n);
    int herr = 0;
    cudaError_t er = cudaMemcpyAsync(&herr, L.err, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (er == cudaSuccess) er = cudaStreamSynchronize(s);
    if (er != cudaSuccess) return cuda_fail(er, "tridiagonal reduction");
    if (herr) {
        set_error("tridiagonal reduction: grid barrier timed out");
        return BSRG_ERR_CUDA;
    }
    return BSRG_OK;
}

}  // namespace bsrg

// LAPACK DSYTRD (uplo 'L') on the device, as used inside DSYEV
extern "C" int bsrg_dsytrd(bsrg_ctx *c, int n, double *A, int lda, double *d, double *e, double *tau)
{
    using namespace bsrg;
    if (!c || !A || !d || (n > 1 && (!e || !tau)) || n < 0 || lda < (n > 0 ? n : 1)) {
        set_error("bsrg_dsytrd: bad arguments");
        return BSRG_ERR_ARG;
    }
    cudaSetDevice(c->device);
    int rc = ctx_reserve(c, trd_workspace_bytes(n > 0 ? n : 1));
    if (rc != BSRG_OK) return rc;
    rc = trd_reduce(c, n, A, lda, d, e, tau, c->ws);
    if (rc != BSRG_OK) return rc;
    // the error flag exists only once a reduction ran (n >= 2 clears and launches)
    if (n < 2) {
        cudaError_t er = cudaStreamSynchronize(c->stream);
        return er == cudaSuccess ? BSRG_OK : cuda_fail(er, "tridiagonal reduction");
    }
    return trd_check(c->ws, n, c->stream);
}
