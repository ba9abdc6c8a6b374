// Dense symmetric eigensolver for sm_100a: two-stage reduction to tridiagonal
// form, divide and conquer, back-transformation.
//
// The reference's DSYEV (LAP_DSYEV, src/libs/ZCOM/LAPACK_calls.f90:54-76,
// called from diag_hd.f90:312) reduces A = Q T Q^T one column at a time
// (DSYTRD: every column reads the whole trailing matrix, a latency-bound
// matrix-vector product per column on a GPU) and diagonalises T.  Here the
// reduction goes through a band matrix, as in LAPACK's two-stage DSYTRD_2STAGE:
//
//   1. dense -> band (bandwidth NB): per panel of NB columns a Householder QR
//      (one cooperative kernel, the panel in shared memory of a few CTAs, one
//      grid barrier per column), then the two-sided update of the trailing
//      matrix A22 <- (I - V T V^T)^T A22 (I - V T V^T) as FP64 tensor-core
//      GEMMs: X = A22 V, Y = X T - 1/2 V (T^T V^T X T), A22 -= V Y^T + Y V^T
//      (one GEMM of inner size 2 NB over the [V | Y | V] buffer);
//   2. band -> tridiagonal: bulge chasing (sweeps of Householder reflectors of
//      length NB, each annihilating one column and chasing the bulge down the
//      band), one persistent cooperative kernel (syevd2 stage 2 below);
//   3. tridiagonal eigenpairs by divide and conquer (tridiag_dc.cu);
//   4. back-transformation: the stage-2 reflectors (in blocks of NB sweeps) and
//      the stage-1 panels (compact WY, GEMMs), applied to the eigenvectors.
#include <algorithm>
#include <cmath>
#include <vector>

#include <cooperative_groups.h>

#include "ctx.h"
#include "dgemm.h"

namespace bsrg {
namespace {

constexpr int NB = 32;              // bandwidth of the intermediate band matrix
constexpr int PQ_ROWS = 512;        // panel rows held in shared memory per CTA
constexpr int PQ_NT = 256;
constexpr unsigned long long WAIT_NS = 2000000000ull;   // bound of every device-side wait (2 s)

__device__ __forceinline__ unsigned long long gtime()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Grid barrier (all CTAs co-resident: cooperative launch).  bar[0] arrivals,
// bar[1] generation.  A wait longer than WAIT_NS sets *err and every CTA leaves.
__device__ bool grid_sync(unsigned *bar, int *err, unsigned nblocks)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned *vgen = bar + 1;
        const unsigned my = *vgen;
        __threadfence();
        if (atomicAdd(bar, 1u) == nblocks - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            const unsigned long long t0 = gtime();
            while (*vgen == my) {
                if (*(volatile int *)err) break;
                if (gtime() - t0 > WAIT_NS) { atomicExch(err, 1); break; }
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *(volatile int *)err == 0;
}

// ---------------------------------------------------------------------------
// stage 1: panel QR
// ---------------------------------------------------------------------------
struct PanelArgs {
    double *P;          // panel (m x NB), leading dimension ldp: rows j+NB.., columns j..j+NB-1 of A
    long ldp;
    int m, rpc;         // rows, rows per CTA
    double *V;          // [V | Y | V] buffer (ld m): V written to columns 0..NB-1 and 2NB..3NB-1
    double *Vs;         // the saved V of this panel for the back-transformation (ld m)
    double *T;          // NB x NB (ld NB), upper triangular
    double *Ts;         // saved copy of T
    double *part;       // per CTA, per column parity: NB dots + NB pivot-row values
    double *gram;       // per CTA: NB x NB Gram partial
    unsigned *bar;
    int *err;
};

// Householder QR of the panel, LAPACK's dgeqrf/dlarfg conventions:
// H_c = I - tau_c v_c v_c^T, v_c(c) = 1, P = H_0 ... H_{NB-1} [R; 0].
__global__ void __launch_bounds__(PQ_NT) panel_qr_kernel(PanelArgs a)
{
    extern __shared__ __align__(16) double ps[];       // rpc x (NB + 1)
    __shared__ double tot[NB], piv[NB], wv[NB], tau_s[NB];
    __shared__ double sc_tau, sc_scale, sc_beta;
    const int cta = blockIdx.x, G = gridDim.x, tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int m = a.m, r0 = cta * a.rpc, nr = max(0, min(a.rpc, m - r0));
    constexpr int LD = NB + 1;
    for (int q = tid; q < nr * NB; q += PQ_NT) {
        const int r = q % nr, c = q / nr;
        ps[r * LD + c] = a.P[(r0 + r) + a.ldp * (long)c];
    }
    const int kb = min(m, NB);
    __syncthreads();
    for (int c = 0; c < kb; c++) {
        double *buf = a.part + ((long)cta * 2 + (c & 1)) * 2 * NB;
        // partial dots over my rows below the pivot: g_k = sum P(r, c) P(r, k), k >= c
        for (int k = c + warp; k < NB; k += PQ_NT / 32) {
            double s = 0.0;
            for (int r = lane; r < nr; r += 32)
                if (r0 + r > c) s += ps[r * LD + c] * ps[r * LD + k];
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) buf[k] = s;
        }
        if (cta == 0)
            for (int k = c + tid; k < NB; k += PQ_NT) buf[NB + k] = ps[c * LD + k];
        __threadfence();
        if (!grid_sync(a.bar, a.err, G)) return;
        for (int k = c + tid; k < NB; k += PQ_NT) {
            double s = 0.0;
            for (int q = 0; q < G; q++) s += __ldcg(a.part + ((long)q * 2 + (c & 1)) * 2 * NB + k);
            tot[k] = s;
            piv[k] = __ldcg(a.part + (c & 1) * 2 * NB + NB + k);
        }
        __syncthreads();
        if (tid == 0) {
            const double alpha = piv[c], sigma = tot[c];
            if (sigma == 0.0) { sc_tau = 0.0; sc_scale = 0.0; sc_beta = alpha; }
            else {
                const double beta = -copysign(sqrt(alpha * alpha + sigma), alpha);
                sc_tau = (beta - alpha) / beta;
                sc_scale = 1.0 / (alpha - beta);
                sc_beta = beta;
            }
            tau_s[c] = sc_tau;
        }
        __syncthreads();
        const double tau = sc_tau, scale = sc_scale;
        for (int k = c + 1 + tid; k < NB; k += PQ_NT) wv[k] = piv[k] + scale * tot[k];   // v^T P(:, k)
        __syncthreads();
        // P(:, k) -= tau v w_k, k > c: rows below the pivot, then the pivot row (CTA 0)
        for (int q = tid; q < nr * (NB - c - 1); q += PQ_NT) {
            const int r = q % nr, k = c + 1 + q / nr;
            if (r0 + r > c) ps[r * LD + k] -= tau * scale * ps[r * LD + c] * wv[k];
        }
        if (cta == 0)
            for (int k = c + 1 + tid; k < NB; k += PQ_NT) ps[c * LD + k] -= tau * wv[k];
        __syncthreads();
        for (int r = tid; r < nr; r += PQ_NT)
            if (r0 + r > c) ps[r * LD + c] *= scale;        // v below the pivot
        if (cta == 0 && tid == 0) ps[c * LD + c] = sc_beta;
        __syncthreads();
    }
    // Gram of V (unit diagonal, zero above), partial over my rows
    double *gp = a.gram + (long)cta * NB * NB;
    for (int q = tid; q < NB * NB; q += PQ_NT) {
        const int i = q % NB, j = q / NB;
        double s = 0.0;
        if (i <= j && j < kb)
            for (int r = 0; r < nr; r++) {
                const int gr = r0 + r;
                const double vi = gr > i ? ps[r * LD + i] : (gr == i ? 1.0 : 0.0);
                const double vj = gr > j ? ps[r * LD + j] : (gr == j ? 1.0 : 0.0);
                s += vi * vj;
            }
        gp[q] = s;
    }
    // V out (unit diagonal, zeros above; columns beyond kb are zero) and the band form of the panel
    for (int q = tid; q < nr * NB; q += PQ_NT) {
        const int r = q % nr, c = q / nr, gr = r0 + r;
        const double v = c < kb ? (gr > c ? ps[r * LD + c] : (gr == c ? 1.0 : 0.0)) : 0.0;
        a.V[gr + (long)m * c] = v;
        a.V[gr + (long)m * (2 * NB + c)] = v;
        a.Vs[gr + (long)m * c] = v;
        a.P[gr + a.ldp * (long)c] = gr <= c ? ps[r * LD + c] : 0.0;
    }
    __threadfence();
    if (!grid_sync(a.bar, a.err, G)) return;
    if (cta != 0) return;
    // T from the Gram matrix: T(c,c) = tau_c, T(0:c, c) = -tau_c T(0:c, 0:c) G(0:c, c)
    double *Gs = ps;                      // reuse: NB x NB
    for (int q = tid; q < NB * NB; q += PQ_NT) {
        double s = 0.0;
        for (int g = 0; g < G; g++) s += __ldcg(a.gram + (long)g * NB * NB + q);
        Gs[q] = s;
    }
    __shared__ double Tt[NB][NB + 1];
    for (int q = tid; q < NB * NB; q += PQ_NT) Tt[q % NB][q / NB] = 0.0;
    __syncthreads();
    for (int c = 0; c < kb; c++) {
        if (tid < c) {
            double s = 0.0;
            for (int l = tid; l < c; l++) s += Tt[tid][l] * Gs[l + NB * c];
            wv[tid] = s;
        }
        __syncthreads();
        if (tid < c) Tt[tid][c] = -tau_s[c] * wv[tid];
        if (tid == 0) Tt[c][c] = tau_s[c];
        __syncthreads();
    }
    for (int q = tid; q < NB * NB; q += PQ_NT) {
        a.T[q] = Tt[q % NB][q / NB];
        a.Ts[q] = Tt[q % NB][q / NB];
    }
}

// The same factorisation on one thread-block cluster (up to 16 CTAs, PQC_ROWS rows each):
// the per-column partial dot products stay in each CTA's shared memory and are read
// by every CTA through distributed shared memory after a hardware cluster barrier,
// instead of a grid barrier over global memory.
constexpr int PQC_ROWS = 640;
constexpr int PQC_MAXG = 16;

__global__ void __launch_bounds__(PQ_NT) panel_qr_cluster_kernel(PanelArgs a)
{
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    extern __shared__ __align__(16) double ps[];       // rpc x (NB + 1) | partials [2][2 NB] | Gram NB x NB
    __shared__ double tot[NB], piv[NB], wv[NB], tau_s[NB];
    __shared__ double sc_tau, sc_scale, sc_beta;
    const int cta = (int)cl.block_rank(), G = (int)cl.num_blocks(), tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int m = a.m, r0 = cta * a.rpc, nr = max(0, min(a.rpc, m - r0));
    constexpr int LD = NB + 1;
    double *part = ps + (size_t)a.rpc * LD;
    double *gram = part + 4 * NB;
    for (int c = warp; c < NB; c += PQ_NT / 32)
        for (int r = lane; r < nr; r += 32) ps[r * LD + c] = a.P[(r0 + r) + a.ldp * (long)c];
    const int kb = min(m, NB);
    __syncthreads();
    for (int c = 0; c < kb; c++) {
        double *buf = part + (c & 1) * 2 * NB;
        for (int k = c + warp; k < NB; k += PQ_NT / 32) {
            double s = 0.0;
            for (int r = lane; r < nr; r += 32)
                if (r0 + r > c) s += ps[r * LD + c] * ps[r * LD + k];
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) buf[k] = s;
        }
        if (cta == 0)
            for (int k = c + tid; k < NB; k += PQ_NT) buf[NB + k] = ps[c * LD + k];
        cl.sync();
        for (int k = c + tid; k < NB; k += PQ_NT) {
            double s = 0.0;
            for (int q = 0; q < G; q++) s += cl.map_shared_rank(buf, q)[k];
            tot[k] = s;
            piv[k] = cl.map_shared_rank(buf, 0)[NB + k];
        }
        __syncthreads();
        if (tid == 0) {
            const double alpha = piv[c], sigma = tot[c];
            if (sigma == 0.0) { sc_tau = 0.0; sc_scale = 0.0; sc_beta = alpha; }
            else {
                const double beta = -copysign(sqrt(alpha * alpha + sigma), alpha);
                sc_tau = (beta - alpha) / beta;
                sc_scale = 1.0 / (alpha - beta);
                sc_beta = beta;
            }
            tau_s[c] = sc_tau;
        }
        __syncthreads();
        const double tau = sc_tau, scale = sc_scale;
        for (int k = c + 1 + tid; k < NB; k += PQ_NT) wv[k] = piv[k] + scale * tot[k];
        __syncthreads();
        // a thread per row (stride 33 doubles: conflict-free), columns k > c in registers' reach
        const double ts_ = tau * scale;
        for (int r = tid; r < nr; r += PQ_NT) {
            if (r0 + r <= c) continue;
            double *row = ps + r * LD;
            const double f = ts_ * row[c];
            for (int k = c + 1; k < NB; k++) row[k] -= f * wv[k];
        }
        if (cta == 0)
            for (int k = c + 1 + tid; k < NB; k += PQ_NT) ps[c * LD + k] -= tau * wv[k];
        __syncthreads();
        for (int r = tid; r < nr; r += PQ_NT)
            if (r0 + r > c) ps[r * LD + c] *= scale;
        if (cta == 0 && tid == 0) ps[c * LD + c] = sc_beta;
        __syncthreads();
    }
    // V in place (unit diagonal, zeros above; columns beyond kb zero), the R part kept aside
    for (int c = warp; c < NB; c += PQ_NT / 32)
        for (int r = lane; r < nr; r += 32) {
            const int gr = r0 + r;
            const double x = ps[r * LD + c];
            const double v = c < kb ? (gr > c ? x : (gr == c ? 1.0 : 0.0)) : 0.0;
            a.V[gr + (long)m * c] = v;
            a.V[gr + (long)m * (2 * NB + c)] = v;
            a.Vs[gr + (long)m * c] = v;
            a.P[gr + a.ldp * (long)c] = gr <= c ? x : 0.0;
        }
    __syncthreads();
    for (int c = warp; c < NB; c += PQ_NT / 32)
        for (int r = lane; r < nr; r += 32) {
            const int gr = r0 + r;
            ps[r * LD + c] = c < kb ? (gr > c ? ps[r * LD + c] : (gr == c ? 1.0 : 0.0)) : 0.0;
        }
    __syncthreads();
    // Gram partial of V over my rows: warp per (i, j) pairs, lanes over rows
    for (int q = warp; q < NB * NB; q += PQ_NT / 32) {
        const int i = q % NB, j = q / NB;
        double sacc = 0.0;
        if (i <= j)
            for (int r = lane; r < nr; r += 32) sacc += ps[r * LD + i] * ps[r * LD + j];
        for (int o = 16; o > 0; o >>= 1) sacc += __shfl_xor_sync(0xffffffffu, sacc, o);
        if (lane == 0) gram[q] = sacc;
    }
    cl.sync();                                          // every CTA's Gram partial is complete
    if (cta == 0) {
        __shared__ double Gs[NB * NB];
        __shared__ double Tt[NB][NB + 1];
        for (int q = tid; q < NB * NB; q += PQ_NT) {
            double s = 0.0;
            for (int g = 0; g < G; g++) s += cl.map_shared_rank(gram, g)[q];
            Gs[q] = s;
            Tt[q % NB][q / NB] = 0.0;
        }
        __syncthreads();
        for (int c = 0; c < kb; c++) {
            if (tid < c) {
                double s = 0.0;
                for (int l = tid; l < c; l++) s += Tt[tid][l] * Gs[l + NB * c];
                wv[tid] = s;
            }
            __syncthreads();
            if (tid < c) Tt[tid][c] = -tau_s[c] * wv[tid];
            if (tid == 0) Tt[c][c] = tau_s[c];
            __syncthreads();
        }
        for (int q = tid; q < NB * NB; q += PQ_NT) {
            a.T[q] = Tt[q % NB][q / NB];
            a.Ts[q] = Tt[q % NB][q / NB];
        }
    }
    cl.sync();                                          // CTA 0 has read every Gram partial
}

// Y = X T (rows), partial M = V^T Y per chunk of 128 rows.  X, V, Y: ld m.
__global__ void __launch_bounds__(128) ypass1_kernel(int m, const double *__restrict__ X, const double *__restrict__ V,
                                                     const double *__restrict__ T, double *Y, double *Mp,
                                                     unsigned *tick)
{
    __shared__ double Ts[NB][NB + 1];
    extern __shared__ __align__(16) double ysm[];        // Vs, Ys: 128 x (NB + 1) each
    double (*Vs)[NB + 1] = (double (*)[NB + 1])ysm;
    double (*Ys)[NB + 1] = (double (*)[NB + 1])(ysm + 128 * (NB + 1));
    const int tid = threadIdx.x, r0 = blockIdx.x * 128, r = r0 + tid;
    for (int q = tid; q < NB * NB; q += 128) Ts[q % NB][q / NB] = T[q];
    __syncthreads();
    double x[NB];
#pragma unroll
    for (int k = 0; k < NB; k++) x[k] = r < m ? X[r + (long)m * k] : 0.0;
#pragma unroll
    for (int c = 0; c < NB; c++) {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < NB; k++) s += x[k] * Ts[k][c];
        Ys[tid][c] = s;
        Vs[tid][c] = r < m ? V[r + (long)m * c] : 0.0;
        if (r < m) Y[r + (long)m * c] = s;
    }
    __syncthreads();
    for (int q = tid; q < NB * NB; q += 128) {
        const int i = q % NB, j = q / NB;
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;     // four chains over the rows
#pragma unroll 4
        for (int rr = 0; rr < 128; rr += 4) {
            s0 = fma(Vs[rr][i], Ys[rr][j], s0);
            s1 = fma(Vs[rr + 1][i], Ys[rr + 1][j], s1);
            s2 = fma(Vs[rr + 2][i], Ys[rr + 2][j], s2);
            s3 = fma(Vs[rr + 3][i], Ys[rr + 3][j], s3);
        }
        Mp[(long)blockIdx.x * NB * NB + q] = (s0 + s1) + (s2 + s3);
    }
    // the last CTA to finish sums the partials in chunk order and forms M2 = 1/2 T^T M once
    // (at Mp + gridDim.x NB^2) for ypass2; it resets the ticket for the next panel
    __shared__ unsigned ticket;
    __threadfence();
    __syncthreads();
    if (tid == 0) ticket = atomicAdd(tick, 1u);
    __syncthreads();
    if (ticket != gridDim.x - 1) return;
    __threadfence();
    double (*Ms)[NB + 1] = Vs;                     // reuse
    for (int q = tid; q < NB * NB; q += 128) {
        double s = 0.0;
        for (int ch = 0; ch < (int)gridDim.x; ch++) s += __ldcg(Mp + (long)ch * NB * NB + q);
        Ms[q % NB][q / NB] = s;
    }
    __syncthreads();
    double *M2 = Mp + (long)gridDim.x * NB * NB;
    for (int q = tid; q < NB * NB; q += 128) {
        const int i = q % NB, j = q / NB;
        double s = 0.0;
        for (int l = 0; l <= i; l++) s += Ts[l][i] * Ms[l][j];     // T upper: T^T(i,l) = T(l,i), l <= i
        M2[q] = 0.5 * s;                                            // column-major M2(i, j)
    }
    if (tid == 0) *tick = 0u;
}

// Y -= V M2 (rows), M2 formed by the last CTA of ypass1
__global__ void __launch_bounds__(128) ypass2_kernel(int m, const double *__restrict__ V, const double *__restrict__ M2g,
                                                     double *Y)
{
    __shared__ double M2[NB][NB + 1];
    const int tid = threadIdx.x;
    for (int q = tid; q < NB * NB; q += 128) M2[q % NB][q / NB] = M2g[q];
    __syncthreads();
    const int r = blockIdx.x * 128 + tid;
    if (r >= m) return;
    double v[NB];
#pragma unroll
    for (int k = 0; k < NB; k++) v[k] = V[r + (long)m * k];
#pragma unroll
    for (int c = 0; c < NB; c++) {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < NB; k++) s += v[k] * M2[k][c];
        Y[r + (long)m * c] -= s;
    }
}

constexpr int YP1_SMEM = 2 * 128 * (NB + 1) * (int)sizeof(double);

// AB[d + 2NB c] = A(c + d, c), d < 2NB (rows beyond the band zero: room for the bulges)
__global__ void band_extract_kernel(int n, const double *__restrict__ A, long lda, double *AB)
{
    const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (idx >= (long)n * 2 * NB) return;
    const int d = (int)(idx % (2 * NB)), c = (int)(idx / (2 * NB));
    AB[idx] = (d <= NB && c + d < n) ? A[(c + d) + lda * (long)c] : 0.0;
}

// ---------------------------------------------------------------------------
// stage 2: band -> tridiagonal (bulge chasing)
// ---------------------------------------------------------------------------
// Band storage: A(r, c), r >= c, r - c < 2NB, at AB[(r - c) + 2NB c] (the NB rows
// below the band hold the bulges).  Sweep j annihilates column j below the
// subdiagonal and chases the bulge: task (j, i) has the window rows
// r0 = j + 1 + i NB .. r1 = min(r0 + NB, n) - 1 and reduces column col (= j for
// i = 0, the previous window's first column otherwise) with one reflector H,
// applied from the left to the rest of the previous bulge (columns col+1..r0-1),
// from both sides to the diagonal block, and from the right to the NB rows
// below the window (creating the next bulge).  Task (j, i) may run once sweep
// j-1 has completed step i+2 (their footprints are disjoint from then on).
constexpr int LDAB = 2 * NB;

__host__ __device__ __forceinline__ int sweep_steps(int n, int j) { return j <= n - 3 ? (n - 3 - j) / NB + 1 : 0; }

struct Sb2stArgs {
    double *AB;
    int n;
    double *V2;        // reflectors: V2[((long)j * S + i) * NB + t]
    double *tau2;      // tau2[(long)j * S + i]
    int S;
    int *progress;     // completed steps per sweep (zero on entry)
    int *err;
};

// one warp per worker CTA; workers take sweeps j = blockIdx.x, + gridDim.x, ...
__global__ void __launch_bounds__(32) sb2st_kernel(Sb2stArgs a)
{
    __shared__ double Lb[NB][NB + 1], Ds[NB][NB + 1], Bs[NB][NB + 1];
    __shared__ double vs[NB], ws_[NB];
    const int t = threadIdx.x, n = a.n;
    double *AB = a.AB;
    auto at = [&](int r, int c) -> double * { return AB + (r - c) + (long)LDAB * c; };
    for (int j = blockIdx.x; j < n - 2; j += gridDim.x) {
        const int nst = sweep_steps(n, j);
        const int nprev = j > 0 ? sweep_steps(n, j - 1) : 0;
        for (int i = 0; i < nst; i++) {
            if (j > 0) {
                const int need = min(i + 3, nprev);
                if (t == 0) {
                    volatile int *pg = a.progress + (j - 1);
                    const unsigned long long t0 = gtime();
                    while (*pg < need) {
                        if (*(volatile int *)a.err) break;
                        if (gtime() - t0 > WAIT_NS) { atomicExch(a.err, 2); break; }
                    }
                    __threadfence();
                }
                __syncwarp();
                if (*(volatile int *)a.err) return;
            }
            const int r0 = j + 1 + i * NB, r1 = min(r0 + NB, n), L = r1 - r0;
            const int col = i == 0 ? j : r0 - NB;
            const int nl = r0 - col - 1;                        // left columns col+1 .. r0-1
            const int r2 = min(r1 + NB, n), nb2 = r2 - r1;      // rows below the window
            // ---- loads (through L2: other workers write the band), every load of a block
            // issued before any is used so their latencies overlap ----
            const double x = t < L ? __ldcg(at(r0 + t, col)) : 0.0;
            {
                double rl[NB - 1], rd[NB], rb[NB];
#pragma unroll
                for (int c = 0; c < NB - 1; c++) rl[c] = (c < nl && t < L) ? __ldcg(at(r0 + t, col + 1 + c)) : 0.0;
#pragma unroll
                for (int a2 = 0; a2 < NB; a2++) rd[a2] = (a2 < L && t < L && a2 >= t) ? __ldcg(at(r0 + a2, r0 + t)) : 0.0;
#pragma unroll
                for (int q = 0; q < NB; q++) rb[q] = (q < nb2 && t < L) ? __ldcg(at(r1 + q, r0 + t)) : 0.0;
#pragma unroll
                for (int c = 0; c < NB - 1; c++) Lb[t][c] = rl[c];
#pragma unroll
                for (int a2 = 0; a2 < NB; a2++) Ds[a2][t] = rd[a2];
#pragma unroll
                for (int q = 0; q < NB; q++) Bs[q][t] = rb[q];
            }
            // ---- the reflector ----
            double sig = (t >= 1 && t < L) ? x * x : 0.0;
            for (int o = 16; o > 0; o >>= 1) sig += __shfl_xor_sync(0xffffffffu, sig, o);
            const double alpha = __shfl_sync(0xffffffffu, x, 0);
            double tau = 0.0, scale = 0.0, beta = alpha;
            if (sig != 0.0) {
                beta = -copysign(sqrt(alpha * alpha + sig), alpha);
                tau = (beta - alpha) / beta;
                scale = 1.0 / (alpha - beta);
            }
            const double v = t == 0 ? 1.0 : (t < L ? x * scale : 0.0);
            vs[t] = v;
            a.V2[((long)j * a.S + i) * NB + t] = v;
            if (t == 0) a.tau2[(long)j * a.S + i] = tau;
            if (t < L) *at(r0 + t, col) = t == 0 ? beta : 0.0;
            __syncwarp();
            if (tau != 0.0) {
                // left: columns col+1 .. r0-1 of the window rows (lane = column)
                if (t < nl) {
                    double w = 0.0;
                    for (int q = 0; q < L; q++) w += vs[q] * Lb[q][t];
                    for (int q = 0; q < L; q++) Lb[q][t] -= tau * vs[q] * w;
                }
                // two-sided on the diagonal block: p = tau D v, w = p - tau/2 (v^T p) v
                double p = 0.0;
                if (t < L)
                    for (int b = 0; b < L; b++) p += (t >= b ? Ds[t][b] : Ds[b][t]) * vs[b];
                p *= tau;
                double vp = v * p;
                for (int o = 16; o > 0; o >>= 1) vp += __shfl_xor_sync(0xffffffffu, vp, o);
                ws_[t] = p - 0.5 * tau * vp * v;
                __syncwarp();
                if (t < L)
                    for (int a2 = t; a2 < L; a2++) Ds[a2][t] -= vs[a2] * ws_[t] + ws_[a2] * vs[t];
                // right: rows below the window (lane = row)
                if (t < nb2) {
                    double sr = 0.0;
                    for (int c = 0; c < L; c++) sr += Bs[t][c] * vs[c];
                    for (int c = 0; c < L; c++) Bs[t][c] -= tau * sr * vs[c];
                }
                __syncwarp();
                // ---- stores ----
                for (int c = 0; c < nl; c++)
                    if (t < L) *at(r0 + t, col + 1 + c) = Lb[t][c];
                for (int a2 = 0; a2 < L; a2++)
                    if (t < L && a2 >= t) *at(r0 + a2, r0 + t) = Ds[a2][t];
                for (int q = 0; q < nb2; q++)
                    if (t < L) *at(r1 + q, r0 + t) = Bs[q][t];
            }
            __threadfence();
            __syncwarp();
            if (t == 0) *(volatile int *)(a.progress + j) = i + 1;
        }
    }
}

// The same tasks with every block held row-wise in registers (lane = row, so the
// band is read and written coalesced), the reductions across rows through shared
// memory, and the x column and left block of step i > 0 taken from step i-1's
// updated lower block (the same rows and columns; no other sweep writes them in
// between: sweep j-1 is at least three steps ahead, sweep j+1 behind).
// K warps per CTA: CTA b takes the groups of K consecutive sweeps g = b, b + gridDim.x, ...,
// warp w sweep g K + w.  A warp waits for its predecessor sweep through a counter in shared
// memory when the predecessor is a warp of the same CTA (w > 0) and through the global
// progress array otherwise; the band itself is exchanged through global memory (L2) as before.
constexpr int SB_WSM = 2 * NB * (NB + 1) + 2 * NB;       // doubles of shared memory per warp

template <int K>
__global__ void __launch_bounds__(32 * K) sb2st2_kernel(Sb2stArgs a)
{
    extern __shared__ __align__(16) double sbsm[];
    __shared__ volatile int sprog[K];          // it * 4096 + completed steps of warp w's sweep
    const int t = threadIdx.x & 31, w = threadIdx.x >> 5, n = a.n;
    double (*Ts)[NB + 1] = (double (*)[NB + 1])(sbsm + w * SB_WSM);            // transpose of D
    double (*Cs)[NB + 1] = (double (*)[NB + 1])(sbsm + w * SB_WSM + NB * (NB + 1));   // carried block
    double *vs = sbsm + w * SB_WSM + 2 * NB * (NB + 1), *ws2 = vs + NB;
    double *AB = a.AB;
    if (threadIdx.x < K) sprog[threadIdx.x] = 0;
    __syncthreads();
    int it = 0;
    auto at = [&](int r, int c) -> double * { return AB + (r - c) + (long)LDAB * c; };
    // wait until sweep j-1 has completed `need` steps (bounded; false: give up, the flag is set)
    auto wait_prev = [&](int j, int need) -> bool {
        if (j > 0 && need > 0) {
            if (t == 0) {
                const unsigned long long t0 = gtime();
                if (w > 0) {
                    const int target = it * 4096 + need;
                    while (sprog[w - 1] < target) {
                        if (*(volatile int *)a.err) break;
                        if (gtime() - t0 > WAIT_NS) { atomicExch(a.err, 2); break; }
                    }
                } else {
                    volatile int *pg = a.progress + (j - 1);
                    while (*pg < need) {
                        if (*(volatile int *)a.err) break;
                        if (gtime() - t0 > WAIT_NS) { atomicExch(a.err, 2); break; }
                    }
                }
                __threadfence();
            }
            __syncwarp();
            if (*(volatile int *)a.err) return false;
        }
        return true;
    };
    // the diagonal and lower blocks of step i of sweep j, lane = row
    auto load_blocks = [&](int j, int i, double *Dr, double *Br) {
        const int r0 = j + 1 + i * NB, r1 = min(r0 + NB, n), L = r1 - r0;
        const int r2 = min(r1 + NB, n), nb2 = r2 - r1;
#pragma unroll
        for (int c = 0; c < NB; c++) Dr[c] = (t < L && c <= t) ? __ldcg(at(r0 + t, r0 + c)) : 0.0;
#pragma unroll
        for (int c = 0; c < NB; c++) Br[c] = (t < nb2 && c < L) ? __ldcg(at(r1 + t, r0 + c)) : 0.0;
    };
    for (int g = blockIdx.x; g * K < n - 2; g += gridDim.x, it++) {
        const int j = g * K + w;
        if (j >= n - 2) break;
        const int nst = sweep_steps(n, j);
        const int nprev = j > 0 ? sweep_steps(n, j - 1) : 0;
        double Dr[NB], Br[NB];
        if (!wait_prev(j, min(3, nprev))) return;
        load_blocks(j, 0, Dr, Br);
        for (int i = 0; i < nst; i++) {
            const int r0 = j + 1 + i * NB, r1 = min(r0 + NB, n), L = r1 - r0;
            const int col = i == 0 ? j : r0 - NB;
            const int nl = r0 - col - 1;
            const int r2 = min(r1 + NB, n), nb2 = r2 - r1;
            // the blocks of this step were loaded at the end of the previous one (or above)
            const double xl = i == 0 ? (t < L ? __ldcg(at(r0 + t, col)) : 0.0) : Cs[t][0];
            // ---- the reflector ----
            double sig = (t >= 1 && t < L) ? xl * xl : 0.0;
            for (int o = 16; o > 0; o >>= 1) sig += __shfl_xor_sync(0xffffffffu, sig, o);
            const double alpha = __shfl_sync(0xffffffffu, xl, 0);
            double tau = 0.0, scale = 0.0, beta = alpha;
            if (sig != 0.0) {
                beta = -copysign(sqrt(alpha * alpha + sig), alpha);
                tau = (beta - alpha) / beta;
                scale = 1.0 / (alpha - beta);
            }
            const double v = t == 0 ? 1.0 : (t < L ? xl * scale : 0.0);
            vs[t] = v;
            a.V2[((long)j * a.S + i) * NB + t] = v;
            if (t == 0) a.tau2[(long)j * a.S + i] = tau;
            if (t < L) *at(r0 + t, col) = t == 0 ? beta : 0.0;
            __syncwarp();
            if (tau != 0.0) {
                // left: columns col+1 .. r0-1 = columns 1.. of the carried block; w_c across rows
                if (nl > 0) {
                    if (t < nl) {
                        double w0 = 0.0, w1 = 0.0;
#pragma unroll
                        for (int q = 0; q < NB; q += 2) {
                            w0 = fma(vs[q], Cs[q][t + 1], w0);
                            w1 = fma(vs[q + 1], Cs[q + 1][t + 1], w1);
                        }
                        ws2[t] = tau * (w0 + w1);
                    }
                    __syncwarp();
                    if (t < L) {
#pragma unroll
                        for (int c = 0; c < NB - 1; c++)
                            if (c < nl) *at(r0 + t, col + 1 + c) = fma(-v, ws2[c], Cs[t][c + 1]);
                    }
                    __syncwarp();
                }
                // two-sided on the diagonal block: p = tau D v, w = p - tau/2 (v^T p) v
#pragma unroll
                for (int c = 0; c < NB; c++) Ts[t][c] = Dr[c];
                __syncwarp();
                double p0 = 0.0, p1 = 0.0;
#pragma unroll
                for (int c = 0; c < NB; c += 2) {
                    const double d0 = c <= t ? Dr[c] : Ts[c][t];           // D(t, c) from the lower triangle
                    const double d1 = c + 1 <= t ? Dr[c + 1] : Ts[c + 1][t];
                    p0 = fma(d0, vs[c], p0);
                    p1 = fma(d1, vs[c + 1], p1);
                }
                const double p = t < L ? tau * (p0 + p1) : 0.0;
                double vp = v * p;
                for (int o = 16; o > 0; o >>= 1) vp += __shfl_xor_sync(0xffffffffu, vp, o);
                const double w = p - 0.5 * tau * vp * v;
                ws2[t] = w;
                __syncwarp();
#pragma unroll
                for (int c = 0; c < NB; c++)
                    if (c <= t) Dr[c] -= v * ws2[c] + w * vs[c];
                // right: rows below the window, s_q = sum_c B(q, c) v_c
                double s0 = 0.0, s1 = 0.0;
#pragma unroll
                for (int c = 0; c < NB; c += 2) {
                    s0 = fma(Br[c], vs[c], s0);
                    s1 = fma(Br[c + 1], vs[c + 1], s1);
                }
                const double sr = tau * (s0 + s1);
#pragma unroll
                for (int c = 0; c < NB; c++) Br[c] = fma(-sr, vs[c], Br[c]);
                // ---- stores, lane = row ----
                if (t < L) {
#pragma unroll
                    for (int c = 0; c < NB; c++)
                        if (c <= t) *at(r0 + t, r0 + c) = Dr[c];
                }
                if (t < nb2) {
#pragma unroll
                    for (int c = 0; c < NB; c++)
                        if (c < L) *at(r1 + t, r0 + c) = Br[c];
                }
            }
            // the next window's x column and left block are this step's lower block
#pragma unroll
            for (int c = 0; c < NB; c++) Cs[t][c] = Br[c];
            // the next step's blocks (written by nobody in this step; sweep j-1 must be three steps
            // ahead of it) are requested before this step's stores are fenced, so the two overlap
            if (i + 1 < nst) {
                if (!wait_prev(j, min(i + 4, nprev))) return;
                load_blocks(j, i + 1, Dr, Br);
            }
            __threadfence();
            __syncwarp();
            if (t == 0) {
                *(volatile int *)(a.progress + j) = i + 1;
                sprog[w] = it * 4096 + i + 1;
            }
        }
    }
}

// The register form with a helper warp: warp 0 computes and stores each step, warp 1 publishes
// the step (fence, then the progress counter) and polls the previous sweep's counter, so that
// neither the release fence nor the poll's round trip to L2 sits between two steps of warp 0.
// Warp 0 hands a step over through the shared counter `done` after a block-scope fence; warp 1
// observes it, and its device-scope fence orders warp 0's stores before the progress counter
// (the fence is cumulative over what warp 1 has observed).  The previous sweep's progress goes
// the other way: warp 1 reads it, fences, and posts it in `seen`.  (A sleep between polls, of
// even 8 ns, measured slower: the sleep's granularity is coarse.)
__global__ void __launch_bounds__(64) sb2st3_kernel(Sb2stArgs a)
{
    __shared__ double Ts[NB][NB + 1], Cs[NB][NB + 1];
    __shared__ double vs[NB], ws2[NB];
    __shared__ volatile int done, seen, quit;
    const int t = threadIdx.x & 31, w = threadIdx.x >> 5, n = a.n;
    double *AB = a.AB;
    auto at = [&](int r, int c) -> double * { return AB + (r - c) + (long)LDAB * c; };
    for (int j = blockIdx.x; j < n - 2; j += gridDim.x) {
        const int nst = sweep_steps(n, j);
        const int nprev = j > 0 ? sweep_steps(n, j - 1) : 0;
        if (threadIdx.x == 0) { done = 0; seen = j > 0 ? 0 : 1 << 30; quit = 0; }
        __syncthreads();
        if (w == 1) {
            // ---- helper: publish warp 0's steps, watch the previous sweep ----
            if (t == 0) {
                int pub = 0, sv = j > 0 ? 0 : 1 << 30;
                unsigned long long t0 = gtime();
                while (pub < nst) {
                    const int d = done;
                    if (d > pub) {
                        __threadfence();
                        *(volatile int *)(a.progress + j) = d;
                        pub = d;
                        t0 = gtime();
                        continue;
                    }
                    if (quit) break;
                    if (sv < nprev) {
                        const int v = *(volatile int *)(a.progress + (j - 1));
                        if (v > sv) {
                            __threadfence();
                            sv = v;
                            seen = v;
                            t0 = gtime();
                            continue;
                        }
                    }
                    if (*(volatile int *)a.err) { quit = 1; break; }
                    if (gtime() - t0 > WAIT_NS) { atomicExch(a.err, 2); quit = 1; break; }
                }
            }
            __syncthreads();
            if (*(volatile int *)a.err) return;
            continue;
        }
        // ---- warp 0: the steps ----
        // wait until the helper has seen the previous sweep complete `need` steps
        auto wait_prev = [&](int need) -> bool {
            if (t == 0) {
                const unsigned long long t0 = gtime();
                while (seen < need) {
                    if (quit) break;
                    if (gtime() - t0 > WAIT_NS) { atomicExch(a.err, 2); quit = 1; break; }
                }
                __threadfence_block();
            }
            __syncwarp();
            return !quit;
        };
        auto load_blocks = [&](int i, double *Dr, double *Br) {
            const int r0 = j + 1 + i * NB, r1 = min(r0 + NB, n), L = r1 - r0;
            const int r2 = min(r1 + NB, n), nb2 = r2 - r1;
#pragma unroll
            for (int c = 0; c < NB; c++) Dr[c] = (t < L && c <= t) ? __ldcg(at(r0 + t, r0 + c)) : 0.0;
#pragma unroll
            for (int c = 0; c < NB; c++) Br[c] = (t < nb2 && c < L) ? __ldcg(at(r1 + t, r0 + c)) : 0.0;
        };
        double Dr[NB], Br[NB];
        bool ok = wait_prev(min(3, nprev));
        if (ok) load_blocks(0, Dr, Br);
        for (int i = 0; ok && i < nst; i++) {
            const int r0 = j + 1 + i * NB, r1 = min(r0 + NB, n), L = r1 - r0;
            const int col = i == 0 ? j : r0 - NB;
            const int nl = r0 - col - 1;
            const int r2 = min(r1 + NB, n), nb2 = r2 - r1;
            const double xl = i == 0 ? (t < L ? __ldcg(at(r0 + t, col)) : 0.0) : Cs[t][0];
            // ---- the reflector ----
            double sig = (t >= 1 && t < L) ? xl * xl : 0.0;
            for (int o = 16; o > 0; o >>= 1) sig += __shfl_xor_sync(0xffffffffu, sig, o);
            const double alpha = __shfl_sync(0xffffffffu, xl, 0);
            double tau = 0.0, scale = 0.0, beta = alpha;
            if (sig != 0.0) {
                beta = -copysign(sqrt(alpha * alpha + sig), alpha);
                tau = (beta - alpha) / beta;
                scale = 1.0 / (alpha - beta);
            }
            const double v = t == 0 ? 1.0 : (t < L ? xl * scale : 0.0);
            vs[t] = v;
            a.V2[((long)j * a.S + i) * NB + t] = v;
            if (t == 0) a.tau2[(long)j * a.S + i] = tau;
            if (t < L) *at(r0 + t, col) = t == 0 ? beta : 0.0;
            __syncwarp();
            if (tau != 0.0) {
                if (nl > 0) {
                    if (t < nl) {
                        double w0 = 0.0, w1 = 0.0;
#pragma unroll
                        for (int q = 0; q < NB; q += 2) {
                            w0 = fma(vs[q], Cs[q][t + 1], w0);
                            w1 = fma(vs[q + 1], Cs[q + 1][t + 1], w1);
                        }
                        ws2[t] = tau * (w0 + w1);
                    }
                    __syncwarp();
                    if (t < L) {
#pragma unroll
                        for (int c = 0; c < NB - 1; c++)
                            if (c < nl) *at(r0 + t, col + 1 + c) = fma(-v, ws2[c], Cs[t][c + 1]);
                    }
                    __syncwarp();
                }
#pragma unroll
                for (int c = 0; c < NB; c++) Ts[t][c] = Dr[c];
                __syncwarp();
                double p0 = 0.0, p1 = 0.0;
#pragma unroll
                for (int c = 0; c < NB; c += 2) {
                    const double d0 = c <= t ? Dr[c] : Ts[c][t];
                    const double d1 = c + 1 <= t ? Dr[c + 1] : Ts[c + 1][t];
                    p0 = fma(d0, vs[c], p0);
                    p1 = fma(d1, vs[c + 1], p1);
                }
                const double p = t < L ? tau * (p0 + p1) : 0.0;
                double vp = v * p;
                for (int o = 16; o > 0; o >>= 1) vp += __shfl_xor_sync(0xffffffffu, vp, o);
                const double wv = p - 0.5 * tau * vp * v;
                ws2[t] = wv;
                __syncwarp();
#pragma unroll
                for (int c = 0; c < NB; c++)
                    if (c <= t) Dr[c] -= v * ws2[c] + wv * vs[c];
                double s0 = 0.0, s1 = 0.0;
#pragma unroll
                for (int c = 0; c < NB; c += 2) {
                    s0 = fma(Br[c], vs[c], s0);
                    s1 = fma(Br[c + 1], vs[c + 1], s1);
                }
                const double sr = tau * (s0 + s1);
#pragma unroll
                for (int c = 0; c < NB; c++) Br[c] = fma(-sr, vs[c], Br[c]);
                if (t < L) {
#pragma unroll
                    for (int c = 0; c < NB; c++)
                        if (c <= t) *at(r0 + t, r0 + c) = Dr[c];
                }
                if (t < nb2) {
#pragma unroll
                    for (int c = 0; c < NB; c++)
                        if (c < L) *at(r1 + t, r0 + c) = Br[c];
                }
            }
#pragma unroll
            for (int c = 0; c < NB; c++) Cs[t][c] = Br[c];
            // hand the step to the helper, then fetch the next step's blocks once the previous sweep
            // is three steps ahead of it
            __threadfence_block();
            __syncwarp();
            if (t == 0) done = i + 1;
            if (i + 1 < nst) {
                ok = wait_prev(min(i + 4, nprev));
                if (ok) load_blocks(i + 1, Dr, Br);
            }
        }
        if (!ok && t == 0) quit = 1;
        __syncthreads();
        if (*(volatile int *)a.err) return;
    }
}

// sb2st3_kernel with each step's two-sided update of the diagonal block and its left update of
// the previous bulge moved to warps of their own (sb2st5_kernel).  Warp 0 keeps the chain from
// step to step -- the reflector from x, the right update of B, and B's new first column as the
// next x -- which reads neither.  Warp 2 loads D of step i itself (once the previous sweep has
// completed step i+2) and updates and stores it; warp 3 applies step i's reflector from the left
// to the previous step's updated B (warp 0 leaves it in one of two shared buffers) and stores
// it; both take v_i and tau_i from a ring of four in shared memory and run behind warp 0.  The
// helper (warp 1) publishes step i once warp 0 has stored step i and warps 2 and 3 step i-1:
// sweep j+1's step i-2, the first to wait for it, reads the first column of D_{i-1} and of the
// previous bulge but neither D_i nor step i's left update.  The arithmetic is sb2st3's.
__global__ void __launch_bounds__(128) sb2st5_kernel(Sb2stArgs a)
{
    __shared__ double Ts[NB][NB + 1], Cs[2][NB][NB + 1], Bsm[2][NB][NB + 1];
    __shared__ double vring[4][NB], tauring[4], ws2[NB], wsd[NB];
    __shared__ volatile int done, doneD, doneL, vready, bready, seen, quit;
    const int t = threadIdx.x & 31, w = threadIdx.x >> 5, n = a.n;
    double *AB = a.AB;
    auto at = [&](int r, int c) -> double * { return AB + (r - c) + (long)LDAB * c; };
    // bounded wait of lane 0 until *flag >= need (false: gave up; the error flag is set)
    auto wait_ge = [&](volatile int *flag, int need) -> bool {
        if (t == 0) {
            const unsigned long long t0 = gtime();
            while (*flag < need) {
                if (quit) break;
                if (gtime() - t0 > WAIT_NS) { atomicExch(a.err, 2); quit = 1; break; }
            }
            __threadfence_block();
        }
        __syncwarp();
        return !quit;
    };
    for (int j = blockIdx.x; j < n - 2; j += gridDim.x) {
        const int nst = sweep_steps(n, j);
        const int nprev = j > 0 ? sweep_steps(n, j - 1) : 0;
        if (threadIdx.x == 0) {
            done = 0; doneD = 0; doneL = 0; vready = 0; bready = 0; seen = j > 0 ? 0 : 1 << 30; quit = 0;
        }
        __syncthreads();
        if (w == 1) {
            // ---- helper: publish what both workers have stored, watch the previous sweep ----
            if (t == 0) {
                int pub = 0, sv = j > 0 ? 0 : 1 << 30;
                unsigned long long t0 = gtime();
                while (pub < nst) {
                    const int d0 = done, dd = doneD, dl = doneL;
                    const int ready = (d0 == nst && dd == nst && dl == nst) ? nst
                                                                          : min(min(d0, min(dd, dl) + 1), nst - 1);
                    if (ready > pub) {
                        __threadfence();
                        *(volatile int *)(a.progress + j) = ready;
                        pub = ready;
                        t0 = gtime();
                        continue;
                    }
                    if (quit) break;
                    if (sv < nprev) {
                        const int v = *(volatile int *)(a.progress + (j - 1));
                        if (v > sv) {
                            __threadfence();
                            sv = v;
                            seen = v;
                            t0 = gtime();
                            continue;
                        }
                    }
                    if (*(volatile int *)a.err) { quit = 1; break; }
                    if (gtime() - t0 > WAIT_NS) { atomicExch(a.err, 2); quit = 1; break; }
                }
            }
        } else if (w == 2) {
            // ---- the diagonal blocks, one step behind warp 0 ----
            for (int i = 0; i < nst; i++) {
                const int r0 = j + 1 + i * NB, r1 = min(r0 + NB, n), L = r1 - r0;
                if (!wait_ge(&seen, min(i + 3, nprev))) break;
                double Dr[NB];
#pragma unroll
                for (int c = 0; c < NB; c++) Dr[c] = (t < L && c <= t) ? __ldcg(at(r0 + t, r0 + c)) : 0.0;
                if (!wait_ge(&vready, i + 1)) break;
                const double *vs = vring[i & 3];
                const double tau = tauring[i & 3], v = vs[t];
                if (tau != 0.0) {
#pragma unroll
                    for (int c = 0; c < NB; c++) Ts[t][c] = Dr[c];
                    __syncwarp();
                    double p0 = 0.0, p1 = 0.0;
#pragma unroll
                    for (int c = 0; c < NB; c += 2) {
                        const double d0 = c <= t ? Dr[c] : Ts[c][t];
                        const double d1 = c + 1 <= t ? Dr[c + 1] : Ts[c + 1][t];
                        p0 = fma(d0, vs[c], p0);
                        p1 = fma(d1, vs[c + 1], p1);
                    }
                    const double p = t < L ? tau * (p0 + p1) : 0.0;
                    double vp = v * p;
                    for (int o = 16; o > 0; o >>= 1) vp += __shfl_xor_sync(0xffffffffu, vp, o);
                    const double wv = p - 0.5 * tau * vp * v;
                    wsd[t] = wv;
                    __syncwarp();
#pragma unroll
                    for (int c = 0; c < NB; c++)
                        if (c <= t) Dr[c] -= v * wsd[c] + wv * vs[c];
                    if (t < L) {
#pragma unroll
                        for (int c = 0; c < NB; c++)
                            if (c <= t) *at(r0 + t, r0 + c) = Dr[c];
                    }
                }
                __threadfence_block();
                __syncwarp();
                if (t == 0) doneD = i + 1;
            }
        } else if (w == 3) {
            // ---- the left updates: step i's reflector on the previous step's updated B; and the
            //      B block of step i+1 into shared buffer (i+1) & 1 for warp 0, once the previous
            //      sweep has completed step i+3 ----
            auto stage_b = [&](int i) -> bool {
                const int r0 = j + 1 + i * NB, r1 = min(r0 + NB, n), L = r1 - r0;
                const int r2 = min(r1 + NB, n), nb2 = r2 - r1;
                if (!wait_ge(&seen, min(i + 3, nprev))) return false;
                double (*B)[NB + 1] = Bsm[i & 1];
#pragma unroll
                for (int c = 0; c < NB; c++) B[t][c] = (t < nb2 && c < L) ? __ldcg(at(r1 + t, r0 + c)) : 0.0;
                __threadfence_block();
                __syncwarp();
                if (t == 0) bready = i + 1;
                return true;
            };
            if (nst > 0 && !stage_b(0)) goto sweep_end;
            for (int i = 0; i < nst; i++) {
                const int r0 = j + 1 + i * NB, r1 = min(r0 + NB, n), L = r1 - r0;
                const int col = i == 0 ? j : r0 - NB;
                const int nl = r0 - col - 1;
                if (!wait_ge(&vready, i + 1)) break;
                const double *vs = vring[i & 3];
                const double tau = tauring[i & 3], v = vs[t];
                if (tau != 0.0 && nl > 0) {
                    double (*C)[NB + 1] = Cs[(i - 1) & 1];
                    if (t < nl) {
                        double w0 = 0.0, w1 = 0.0;
#pragma unroll
                        for (int q = 0; q < NB; q += 2) {
                            w0 = fma(vs[q], C[q][t + 1], w0);
                            w1 = fma(vs[q + 1], C[q + 1][t + 1], w1);
                        }
                        ws2[t] = tau * (w0 + w1);
                    }
                    __syncwarp();
                    if (t < L) {
#pragma unroll
                        for (int c = 0; c < NB - 1; c++)
                            if (c < nl) *at(r0 + t, col + 1 + c) = fma(-v, ws2[c], C[t][c + 1]);
                    }
                    __syncwarp();
                }
                __threadfence_block();
                __syncwarp();
                if (t == 0) doneL = i + 1;
                if (i + 1 < nst && !stage_b(i + 1)) break;
            }
        } else {
            // ---- warp 0: reflectors and right updates ----
            double Br[NB], xnext = 0.0;
            bool ok = wait_ge(&seen, min(3, nprev));
            for (int i = 0; ok && i < nst; i++) {
                const int r0 = j + 1 + i * NB, r1 = min(r0 + NB, n), L = r1 - r0;
                const int col = i == 0 ? j : r0 - NB;
                const int r2 = min(r1 + NB, n), nb2 = r2 - r1;
                const double xl = i == 0 ? (t < L ? __ldcg(at(r0 + t, col)) : 0.0) : xnext;
                // ---- the reflector, into ring slot i & 3 once warp 2 has finished step i-4 ----
                double sig = (t >= 1 && t < L) ? xl * xl : 0.0;
                for (int o = 16; o > 0; o >>= 1) sig += __shfl_xor_sync(0xffffffffu, sig, o);
                const double alpha = __shfl_sync(0xffffffffu, xl, 0);
                double tau = 0.0, scale = 0.0, beta = alpha;
                if (sig != 0.0) {
                    beta = -copysign(sqrt(alpha * alpha + sig), alpha);
                    tau = (beta - alpha) / beta;
                    scale = 1.0 / (alpha - beta);
                }
                const double v = t == 0 ? 1.0 : (t < L ? xl * scale : 0.0);
                if (i >= 4 && (!(ok = wait_ge(&doneD, i - 3)) || !(ok = wait_ge(&doneL, i - 3)))) break;
                double *vs = vring[i & 3];
                vs[t] = v;
                if (t == 0) tauring[i & 3] = tau;
                __threadfence_block();                   // (before the global stores: it need not wait for them)
                __syncwarp();
                if (t == 0) vready = i + 1;
                a.V2[((long)j * a.S + i) * NB + t] = v;
                if (t == 0) a.tau2[(long)j * a.S + i] = tau;
                if (t < L) *at(r0 + t, col) = t == 0 ? beta : 0.0;
                if (!(ok = wait_ge(&bready, i + 1))) break;
                {
                    const double (*B)[NB + 1] = Bsm[i & 1];
#pragma unroll
                    for (int c = 0; c < NB; c++) Br[c] = B[t][c];
                }
                if (tau != 0.0) {
                    double s0 = 0.0, s1 = 0.0;
#pragma unroll
                    for (int c = 0; c < NB; c += 2) {
                        s0 = fma(Br[c], vs[c], s0);
                        s1 = fma(Br[c + 1], vs[c + 1], s1);
                    }
                    const double sr = tau * (s0 + s1);
#pragma unroll
                    for (int c = 0; c < NB; c++) Br[c] = fma(-sr, vs[c], Br[c]);
                    if (t < nb2) {
#pragma unroll
                        for (int c = 0; c < NB; c++)
                            if (c < L) *at(r1 + t, r0 + c) = Br[c];
                    }
                }
                // B goes to buffer i & 1 for warp 3's left update of step i+1, once warp 3 is done
                // with the buffer's last use (step i-1)
                xnext = Br[0];
                if (i >= 1 && !(ok = wait_ge(&doneL, i))) break;
#pragma unroll
                for (int c = 0; c < NB; c++) Cs[i & 1][t][c] = Br[c];
                __threadfence_block();
                __syncwarp();
                if (t == 0) done = i + 1;
            }
            if (!ok && t == 0) quit = 1;
        }
    sweep_end:
        __syncthreads();
        if (*(volatile int *)a.err) return;
    }
}

// d(c) = A(c, c), e(c) = A(c+1, c)
__global__ void tridiag_extract_kernel(int n, const double *__restrict__ AB, double *d, double *e)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    d[c] = AB[(long)LDAB * c];
    if (c + 1 < n) e[c] = AB[1 + (long)LDAB * c];
}

// ---------------------------------------------------------------------------
// back-transformation of the stage-2 reflectors
// ---------------------------------------------------------------------------
// Block (g, i): the step-i reflectors of sweeps j = g NB + q, q < NB, as one
// compact WY factor I - V T V^T = H_{gNB} H_{gNB+1} ... (V column q occupies rows
// q .. q + NB - 1 of the block's window, which starts at row g NB + 1 + i NB).
// Applied to Z: groups g descending, within a group blocks i ascending, each
// block's reflectors in the product order above -- the order of creation
// reversed up to commuting (disjoint) pairs.
__device__ __forceinline__ int q2_nvalid(int n, int g, int i)
{
    int nv = 0;
    for (int q = 0; q < NB; q++) {
        const int j = g * NB + q;
        if (j < n - 2 && i < sweep_steps(n, j)) nv = q + 1;
    }
    return nv;
}

// T factor of every block (one CTA of 32 threads per block)
__global__ void __launch_bounds__(32) q2_tfactor_kernel(int n, int S, const double *__restrict__ V2,
                                                        const double *__restrict__ tau2, double *Tq)
{
    const int g = blockIdx.y, i = blockIdx.x, t = threadIdx.x;
    double *T = Tq + ((long)g * S + i) * NB * NB;
    __shared__ double Vb[2 * NB][NB + 1], Gs[NB][NB + 1], Tt[NB][NB + 1], tau[NB], tmp[NB];
    const int nv = q2_nvalid(n, g, i);
    for (int r = 0; r < 2 * NB; r++) Vb[r][t] = 0.0;
    __syncwarp();
    if (t < nv) {
        const int j = g * NB + t;
        for (int q = 0; q < NB; q++) Vb[t + q][t] = V2[((long)j * S + i) * NB + q];
        tau[t] = tau2[(long)j * S + i];
    } else tau[t] = 0.0;
    __syncwarp();
    for (int b = 0; b < NB; b++) {       // Gs[t][b] = V(:, t) . V(:, b)
        double s = 0.0;
        for (int r = 0; r < 2 * NB; r++) s += Vb[r][t] * Vb[r][b];
        Gs[t][b] = s;
        Tt[t][b] = 0.0;
    }
    __syncwarp();
    for (int c = 0; c < nv; c++) {
        if (t < c) {
            double s = 0.0;
            for (int l = t; l < c; l++) s += Tt[t][l] * Gs[l][c];
            tmp[t] = s;
        }
        __syncwarp();
        if (t < c) Tt[t][c] = -tau[c] * tmp[t];
        if (t == 0) Tt[c][c] = tau[c];
        __syncwarp();
    }
    for (int c = 0; c < NB; c++) T[t + NB * c] = Tt[t][c];
}

constexpr int Q2_COLS = 32;
constexpr int Q2_NT = 256;
constexpr int Q2_SMEM = (2 * (2 * NB) * (Q2_COLS + 1) + 2 * NB * (NB + 1)) * (int)sizeof(double);

// Z (n x ncol, ldz) <- Q2 Z; one CTA per strip of Q2_COLS columns
__global__ void __launch_bounds__(Q2_NT) q2_apply_kernel(int n, int S, int ncol, const double *__restrict__ V2,
                                                         const double *__restrict__ Tq, double *Z, long ldz)
{
    extern __shared__ __align__(16) double qsm[];
    double (*Zw)[Q2_COLS + 1] = (double (*)[Q2_COLS + 1])qsm;                    // 2NB rows of the window
    double (*Vb)[Q2_COLS + 1] = (double (*)[Q2_COLS + 1])(qsm + 2 * NB * (Q2_COLS + 1));   // V (2NB x NB)
    double (*Ts)[NB + 1] = (double (*)[NB + 1])(qsm + 4 * NB * (Q2_COLS + 1));
    double (*W)[NB + 1] = (double (*)[NB + 1])(qsm + 4 * NB * (Q2_COLS + 1) + NB * (NB + 1));
    const int tid = threadIdx.x, c0 = blockIdx.x * Q2_COLS;
    const int cl = tid % Q2_COLS, rg = tid / Q2_COLS;        // column, row group (8)
    const int ng = (n - 2 + NB - 1) / NB;
    for (int g = ng - 1; g >= 0; g--) {
        const int imax = sweep_steps(n, g * NB);
        for (int i = 0; i < imax; i++) {
            const int nv = q2_nvalid(n, g, i);
            if (nv == 0) continue;
            const int top = g * NB + 1 + i * NB;
            const int nrow = min(2 * NB - 1, n - top);
            __syncthreads();
            for (int q = tid; q < 2 * NB * NB; q += Q2_NT) {
                const int r = q % (2 * NB), c = q / (2 * NB);
                double v = 0.0;
                if (c < nv && r >= c && r < c + NB) {
                    const int j = g * NB + c;
                    v = V2[((long)j * S + i) * NB + (r - c)];
                }
                Vb[r][c] = v;
            }
            for (int q = tid; q < NB * NB; q += Q2_NT) Ts[q % NB][q / NB] = Tq[((long)g * S + i) * NB * NB + q];
            for (int q = tid; q < 2 * NB * Q2_COLS; q += Q2_NT) {
                const int r = q % (2 * NB), c = q / (2 * NB);
                Zw[r][c] = (r < nrow && c0 + c < ncol) ? Z[(top + r) + ldz * (long)(c0 + c)] : 0.0;
            }
            __syncthreads();
            // W = V^T Zw (NB x cols): thread (cl, rg) computes rows q = rg, rg + 8, ...
            for (int q = rg; q < NB; q += Q2_NT / Q2_COLS) {
                double sacc = 0.0;
                for (int r = q; r < q + NB && r < 2 * NB; r++) sacc += Vb[r][q] * Zw[r][cl];
                W[q][cl] = sacc;
            }
            __syncthreads();
            // W2 = T W (T upper), kept in registers then written back to W
            double w2[NB / (Q2_NT / Q2_COLS)];
#pragma unroll
            for (int k = 0; k < NB / (Q2_NT / Q2_COLS); k++) {
                const int q = rg + k * (Q2_NT / Q2_COLS);
                double sacc = 0.0;
                for (int l = q; l < NB; l++) sacc += Ts[q][l] * W[l][cl];
                w2[k] = sacc;
            }
            __syncthreads();
#pragma unroll
            for (int k = 0; k < NB / (Q2_NT / Q2_COLS); k++) W[rg + k * (Q2_NT / Q2_COLS)][cl] = w2[k];
            __syncthreads();
            // Zw -= V W2
            for (int r = rg; r < nrow; r += Q2_NT / Q2_COLS) {
                double sacc = 0.0;
                const int qlo = max(0, r - NB + 1), qhi = min(NB - 1, r);
                for (int q = qlo; q <= qhi; q++) sacc += Vb[r][q] * W[q][cl];
                if (c0 + cl < ncol) Z[(top + r) + ldz * (long)(c0 + cl)] = Zw[r][cl] - sacc;
            }
        }
    }
}

// Wavefront form of the same application: one CTA per strip of 32 columns, Q2W_WARPS
// warps; warp w applies groups q = w, w + Q2W_WARPS, ... in the order g = ng-1-q, each
// group's blocks ascending.  Block (g, i) overlaps only blocks i-2 .. i of group g+1, so
// it may run once group g+1 has finished block i (or all its blocks): warps wait on the
// previous group's progress in shared memory (bounded), lane = column, each warp keeps its
// block's window in shared memory.
constexpr int Q2W_WARPS = 6;
constexpr int Q2W_SMEM = Q2W_WARPS * (2 * NB) * 33 * (int)sizeof(double);

__global__ void __launch_bounds__(Q2W_WARPS * 32, 2) q2w_apply_kernel(int n, int S, int ncol,
                                                                   const double *__restrict__ V2,
                                                                   const double *__restrict__ Tq, double *Z, long ldz,
                                                                   int *err)
{
    extern __shared__ __align__(16) double q2w_sm[];
    __shared__ volatile int prog[1024];          // blocks done per group (q order), up to 1024 groups
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int c = blockIdx.x * 32 + lane;
    const bool cok = c < ncol;
    double (*Zw)[33] = (double (*)[33])(q2w_sm + wid * (2 * NB) * 33);   // window rows x 32 columns (+pad)
    const int ng = (n - 2 + NB - 1) / NB;
    for (int q = threadIdx.x; q < ng && q < 1024; q += blockDim.x) prog[q] = 0;
    __syncthreads();
    for (int q = wid; q < ng; q += Q2W_WARPS) {
        const int g = ng - 1 - q;
        const int imax = sweep_steps(n, g * NB);
        const int iprev = q > 0 ? sweep_steps(n, (g + 1) * NB) : 0;
        for (int i = 0; i < imax; i++) {
            if (q > 0) {
                const int need = min(i + 1, iprev);
                const unsigned long long t0 = gtime();
                while (prog[q - 1] < need) {
                    if (gtime() - t0 > WAIT_NS) { atomicExch(err, 3); break; }
                }
                __threadfence_block();
            }
            const int nv = q2_nvalid(n, g, i);
            const int top = g * NB + 1 + i * NB;
            const int nrow = min(2 * NB - 1, n - top);
#pragma unroll
            for (int r0w = 0; r0w < 2 * NB; r0w += 16) {     // 16 loads in flight at a time
                double zr[16];
#pragma unroll
                for (int r = 0; r < 16; r++)
                    zr[r] = (cok && r0w + r < nrow) ? Z[(top + r0w + r) + ldz * (long)c] : 0.0;
#pragma unroll
                for (int r = 0; r < 16; r++) Zw[r0w + r][lane] = zr[r];
            }
            __syncwarp();
            // W = V^T Zw, then W2 = T W, then Zw -= V W2 (lane = column)
            const double *Vb = V2 + ((long)(g * NB) * S + i) * NB;     // sweep j = g NB + qq: + qq * S * NB
            const double *T = Tq + ((long)g * S + i) * NB * NB;
            double w[NB];
#pragma unroll
            for (int qq = 0; qq < NB; qq++) {
                double sacc = 0.0;
                if (qq < nv) {
                    const double *v = Vb + (long)qq * S * NB;
#pragma unroll 8
                    for (int t = 0; t < NB; t++) sacc += __ldg(v + t) * Zw[qq + t][lane];
                }
                w[qq] = sacc;
            }
            double w2[NB];
#pragma unroll
            for (int qq = 0; qq < NB; qq++) {
                double sacc = 0.0;
#pragma unroll
                for (int l = qq; l < NB; l++) sacc += __ldg(T + qq + NB * l) * w[l];
                w2[qq] = sacc;
            }
#pragma unroll
            for (int qq = 0; qq < NB; qq++) {
                if (qq < nv) {
                    const double *v = Vb + (long)qq * S * NB;
#pragma unroll 8
                    for (int t = 0; t < NB; t++) Zw[qq + t][lane] -= __ldg(v + t) * w2[qq];
                }
            }
            __syncwarp();
            if (cok)
                for (int r = 0; r < nrow; r++) Z[(top + r) + ldz * (long)c] = Zw[r][lane];
            __threadfence_block();
            __syncwarp();
            if (lane == 0) prog[q] = i + 1;
        }
        if (imax == 0 && lane == 0) prog[q] = 0;
    }
}

// ---------------------------------------------------------------------------
// The same application on the FP64 tensor pipe, with the strip's rows staged in
// shared memory.  One CTA per strip of 32 columns; its Q2R_W warps take the groups
// in rounds: round r gives warp w the group g0 - w (g0 = ng-1 - r Q2R_W), and all
// warps of a round walk down the strip together, warp w one block behind warp w-1
// (block (g, i) waits until group g+1 has finished its block i, as above).  The
// rows between the last warp's window and the first warp's live in a ring of
// Q2R_RING rows: the first warp loads the 32 new rows of each window, the last warp
// writes back the 32 rows it leaves, and the first warp may not run more than
// Q2R_RING / NB - 2 Q2R_W blocks ahead of the last (bounded waits).  So every
// element of Z crosses HBM twice per round instead of twice per block.  A block
// is three tensor-core products on the window (lane fragments of m8n8k4):
//   W = V^T Zw (32 x 64 x 32, the band of V only), W2 = T W (T upper), Zw -= V W2.
// ---------------------------------------------------------------------------
constexpr int Q2R_W = 4;                    // warps (groups per round)
constexpr int Q2R_RING = 256;               // ring rows, a power of two >= 2 NB Q2R_W
constexpr int Q2R_LD = 36;                  // row stride of the ring, of W and of T (4 mod 16 doubles)
constexpr int Q2R_LDV = 37;                 // row stride of a block's V (reflector q: V(q, t) at q LDV + t)
constexpr int Q2R_WARP = NB * (2 * Q2R_LD + Q2R_LDV);   // doubles per warp: W, T, V
constexpr int Q2R_SMEM = (Q2R_RING * Q2R_LD + Q2R_W * Q2R_WARP) * (int)sizeof(double);
static_assert(Q2R_RING >= 2 * NB * Q2R_W && (Q2R_RING & (Q2R_RING - 1)) == 0, "ring size");

__device__ __forceinline__ void q2r_mma(double &d0, double &d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// rows [a, b) of the strip between Z and the ring; 4 rows x 8 columns per 32 threads
template <int RING = Q2R_RING>
__device__ __forceinline__ void q2r_xfer(double *ring, double *Z, long ldz, int n, int c0, int ncl, int a, int b,
                                         bool store, int t0, int nthr)
{
    if (b <= a) return;
    const int nchunk = ((b - a + 3) / 4) * 4;        // chunks of 4 rows x 8 columns
    const int total = nchunk * 32;
    if (store) {
        for (int q = t0; q < total; q += nthr) {
            const int ch = q >> 5, l = q & 31;
            const int row = a + (ch >> 2) * 4 + (l >> 3), col = (ch & 3) * 8 + (l & 7);
            if (row < b && row < n && col < ncl)
                Z[row + ldz * (long)(c0 + col)] = ring[(row & (RING - 1)) * Q2R_LD + col];
        }
        return;
    }
    // loads in batches of 16 per thread, all issued before any is stored
    for (int q0 = t0; q0 < total; q0 += 16 * nthr) {
        double v[16];
#pragma unroll
        for (int u = 0; u < 16; u++) {
            const int q = q0 + u * nthr, ch = q >> 5, l = q & 31;
            const int row = a + (ch >> 2) * 4 + (l >> 3), col = (ch & 3) * 8 + (l & 7);
            v[u] = (q < total && row < b && row < n && col < ncl) ? Z[row + ldz * (long)(c0 + col)] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 16; u++) {
            const int q = q0 + u * nthr, ch = q >> 5, l = q & 31;
            const int row = a + (ch >> 2) * 4 + (l >> 3), col = (ch & 3) * 8 + (l & 7);
            if (q < total && row < b) ring[(row & (RING - 1)) * Q2R_LD + col] = v[u];
        }
    }
}

__global__ void __launch_bounds__(Q2R_W * 32, 1) q2r_apply_kernel(int n, int S, int ncol,
                                                                 const double *__restrict__ V2,
                                                                 const double *__restrict__ Tq, double *Z,
                                                                 long ldz, int *err)
{
    extern __shared__ __align__(16) double q2r_sm[];
    __shared__ volatile int prog[Q2R_W];
    double *ring = q2r_sm;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, lr = lane >> 2, lc = lane & 3;
    double *Wb = q2r_sm + Q2R_RING * Q2R_LD + wid * Q2R_WARP;       // W, then W2
    double *Tsm = Wb + NB * Q2R_LD;                                  // T(q, l) at q + LD l
    double *Vsm = Tsm + NB * Q2R_LD;                                 // V(q, t) at q LDV + t
    const int c0 = blockIdx.x * 32, ncl = min(32, ncol - c0);
    const int ng = (n - 2 + NB - 1) / NB;
    for (int g0 = ng - 1; g0 >= 0; g0 -= Q2R_W) {
        const int gl = max(g0 - Q2R_W + 1, 0), nw = g0 - gl + 1;
        __syncthreads();                              // the previous round's rows are written back
        q2r_xfer(ring, Z, ldz, n, c0, ncl, gl * NB + 1, g0 * NB + 1 + 2 * NB, false, tid, blockDim.x);
        if (tid < Q2R_W) prog[tid] = 0;
        __syncthreads();
        const int ilast = sweep_steps(n, gl * NB);
        if (wid < nw) {
            const int g = g0 - wid;
            const int imax = sweep_steps(n, g * NB);
            const int iprev = wid > 0 ? sweep_steps(n, (g + 1) * NB) : 0;
            for (int i = 0; i < imax; i++) {
                const unsigned long long t0 = gtime();
                if (wid > 0) {
                    const int need = min(i + 1, iprev);
                    while (prog[wid - 1] < need)
                        if (gtime() - t0 > WAIT_NS) { atomicExch(err, 3); break; }
                } else if (nw > 1) {
                    // the ring slots of the new rows must have been written back by the last warp
                    const int need = min(i + nw - Q2R_RING / NB + 1, ilast);
                    while (need > 0 && prog[nw - 1] < need)
                        if (gtime() - t0 > WAIT_NS) { atomicExch(err, 3); break; }
                }
                __threadfence_block();
                const int top = (g + i) * NB + 1;
                const int nrow = min(2 * NB - 1, n - top);
                if (wid == 0 && i > 0) q2r_xfer(ring, Z, ldz, n, c0, ncl, top + NB, top + 2 * NB, false, lane, 32);
                __syncwarp();
                const int nv = q2_nvalid(n, g, i);
                {
                    // the block's reflectors and T into shared memory: 64 coalesced loads per lane in flight
                    const double *Vblk = V2 + ((long)(g * NB) * S + i) * NB;   // reflector q at + q S NB
                    const double *T = Tq + ((long)g * S + i) * NB * NB;
                    double vr[NB], tr[NB];
#pragma unroll
                    for (int q = 0; q < NB; q++) vr[q] = q < nv ? __ldg(Vblk + (long)q * S * NB + lane) : 0.0;
#pragma unroll
                    for (int l = 0; l < NB; l++) tr[l] = __ldg(T + lane + NB * l);
#pragma unroll
                    for (int q = 0; q < NB; q++) Vsm[q * Q2R_LDV + lane] = vr[q];
#pragma unroll
                    for (int l = 0; l < NB; l++) Tsm[lane + Q2R_LD * l] = tr[l];
                }
                __syncwarp();
                // ---- W = V^T Zw: M = q (4 tiles), N = column (4), K = window row (16 steps) ----
                double acc[4][4][2];
#pragma unroll
                for (int a = 0; a < 4; a++)
#pragma unroll
                    for (int b = 0; b < 4; b++) acc[a][b][0] = acc[a][b][1] = 0.0;
#pragma unroll
                for (int ks = 0; ks < 16; ks++) {
                    const int r = 4 * ks + lc;
                    double bz[4];
                    const double *rrow = ring + ((top + r) & (Q2R_RING - 1)) * Q2R_LD;
#pragma unroll
                    for (int nt = 0; nt < 4; nt++) bz[nt] = r < nrow ? rrow[8 * nt + lr] : 0.0;
#pragma unroll
                    for (int mt = 0; mt < 4; mt++) {
                        if (ks < 2 * mt || ks >= 2 * mt + 10) continue;
                        const int q = 8 * mt + lr, t = r - q;
                        const double a = (t >= 0 && t < NB && q < nv && r < nrow) ? Vsm[q * Q2R_LDV + t] : 0.0;
#pragma unroll
                        for (int nt = 0; nt < 4; nt++) q2r_mma(acc[mt][nt][0], acc[mt][nt][1], a, bz[nt]);
                    }
                }
#pragma unroll
                for (int mt = 0; mt < 4; mt++)
#pragma unroll
                    for (int nt = 0; nt < 4; nt++) {
                        Wb[(8 * mt + lr) * Q2R_LD + 8 * nt + 2 * lc] = acc[mt][nt][0];
                        Wb[(8 * mt + lr) * Q2R_LD + 8 * nt + 2 * lc + 1] = acc[mt][nt][1];
                        acc[mt][nt][0] = acc[mt][nt][1] = 0.0;
                    }
                __syncwarp();
                // ---- W2 = T W: M = q, N = column, K = l (T upper: l >= q) ----
#pragma unroll
                for (int ks = 0; ks < 8; ks++) {
                    const int l = 4 * ks + lc;
                    double bw[4];
#pragma unroll
                    for (int nt = 0; nt < 4; nt++) bw[nt] = Wb[l * Q2R_LD + 8 * nt + lr];
#pragma unroll
                    for (int mt = 0; mt < 4; mt++) {
                        if (ks < 2 * mt) continue;
                        const double a = Tsm[(8 * mt + lr) + Q2R_LD * l];
#pragma unroll
                        for (int nt = 0; nt < 4; nt++) q2r_mma(acc[mt][nt][0], acc[mt][nt][1], a, bw[nt]);
                    }
                }
                __syncwarp();
#pragma unroll
                for (int mt = 0; mt < 4; mt++)
#pragma unroll
                    for (int nt = 0; nt < 4; nt++) {
                        Wb[(8 * mt + lr) * Q2R_LD + 8 * nt + 2 * lc] = acc[mt][nt][0];
                        Wb[(8 * mt + lr) * Q2R_LD + 8 * nt + 2 * lc + 1] = acc[mt][nt][1];
                    }
                __syncwarp();
                // ---- Zw -= V W2: M = window row (8 tiles, two halves), N = column, K = q ----
#pragma unroll
                for (int mh = 0; mh < 2; mh++) {
#pragma unroll
                    for (int a = 0; a < 4; a++) {
                        const int r = 8 * (4 * mh + a) + lr;
                        const double *rrow = ring + ((top + r) & (Q2R_RING - 1)) * Q2R_LD;
#pragma unroll
                        for (int nt = 0; nt < 4; nt++) {
                            acc[a][nt][0] = r < nrow ? rrow[8 * nt + 2 * lc] : 0.0;
                            acc[a][nt][1] = r < nrow ? rrow[8 * nt + 2 * lc + 1] : 0.0;
                        }
                    }
#pragma unroll
                    for (int ks = 0; ks < 8; ks++) {
                        const int q = 4 * ks + lc;
                        double bw[4];
#pragma unroll
                        for (int nt = 0; nt < 4; nt++) bw[nt] = Wb[q * Q2R_LD + 8 * nt + lr];
#pragma unroll
                        for (int a = 0; a < 4; a++) {
                            const int mt = 4 * mh + a;
                            const int klo = 2 * mt - 8 > 0 ? 2 * mt - 8 : 0, khi = 2 * mt + 1 < 7 ? 2 * mt + 1 : 7;
                            if (ks < klo || ks > khi) continue;
                            const int r = 8 * mt + lr, t = r - q;
                            const double v = (t >= 0 && t < NB && q < nv && r < nrow) ? Vsm[q * Q2R_LDV + t] : 0.0;
#pragma unroll
                            for (int nt = 0; nt < 4; nt++) q2r_mma(acc[a][nt][0], acc[a][nt][1], -v, bw[nt]);
                        }
                    }
#pragma unroll
                    for (int a = 0; a < 4; a++) {
                        const int r = 8 * (4 * mh + a) + lr;
                        if (r < nrow) {
                            double *rrow = ring + ((top + r) & (Q2R_RING - 1)) * Q2R_LD;
#pragma unroll
                            for (int nt = 0; nt < 4; nt++) {
                                rrow[8 * nt + 2 * lc] = acc[a][nt][0];
                                rrow[8 * nt + 2 * lc + 1] = acc[a][nt][1];
                            }
                        }
                    }
                }
                __syncwarp();
                // the last warp leaves the window's first NB rows for good this round
                if (wid == nw - 1) q2r_xfer(ring, Z, ldz, n, c0, ncl, top, top + NB, true, lane, 32);
                __threadfence_block();
                __syncwarp();
                if (lane == 0) prog[wid] = i + 1;
            }
        }
        __syncthreads();
        // rows below the last warp's last block
        const int rdone = ilast > 0 ? (gl + ilast) * NB + 1 : gl * NB + 1;
        q2r_xfer(ring, Z, ldz, n, c0, ncl, rdone, n, true, tid, blockDim.x);
    }
}

// ---------------------------------------------------------------------------
// The ring application with two warps per group: warp h of a pair owns columns
// 16h .. 16h+15 of the strip, so 8 warps run 4 groups and every scheduler has two
// warps to switch between.  The pair shares its block's reflectors, staged as the
// dense band V(r, q) (r = window row, zeros outside the band and below the window)
// so that no fragment load needs a mask, and T; the two halves depend only on the
// same half of the neighbouring groups (their columns are disjoint).
// ---------------------------------------------------------------------------
constexpr int Q2P_PAIR = (2 * NB + 2 * NB) * Q2R_LD;            // doubles per pair: V band (64 rows), T, W
template <int G, int RING> constexpr int q2p_smem() { return (RING * Q2R_LD + G * Q2P_PAIR) * (int)sizeof(double); }

__device__ __forceinline__ void pair_sync(int p) { asm volatile("bar.sync %0, 64;" ::"r"(p + 1)); }

// rows [a, a + 32) (cut at b) of the 16 columns of half h: chunks of 4 rows x 8 columns, lane l of
// chunk u holds row a + 4 (u >> 1) + (l >> 3), column 16 h + 8 (u & 1) + (l & 7)
__device__ __forceinline__ void q2p_fetch(double (&v)[16], const double *Z, long ldz, int n, int c0, int ncl, int h,
                                          int a, int b, int lane)
{
#pragma unroll
    for (int u = 0; u < 16; u++) {
        const int row = a + (u >> 1) * 4 + (lane >> 3), col = 16 * h + (u & 1) * 8 + (lane & 7);
        v[u] = (row < b && row < n && col < ncl) ? Z[row + ldz * (long)(c0 + col)] : 0.0;
    }
}

template <int RING>
__device__ __forceinline__ void q2p_put(const double (&v)[16], double *ring, int h, int a, int b, int lane)
{
#pragma unroll
    for (int u = 0; u < 16; u++) {
        const int row = a + (u >> 1) * 4 + (lane >> 3), col = 16 * h + (u & 1) * 8 + (lane & 7);
        if (row < b) ring[(row & (RING - 1)) * Q2R_LD + col] = v[u];
    }
}

// rows [a, b) of the 16 columns of half h from the ring back to Z (one warp)
template <int RING>
__device__ __forceinline__ void q2p_store(const double *ring, double *Z, long ldz, int n, int c0, int ncl, int h,
                                          int a, int b, int lane)
{
    if (b <= a) return;
    const int total = ((b - a + 3) / 4) * 2 * 32;      // chunks of 4 rows x 8 columns, 2 column chunks
    for (int q = lane; q < total; q += 32) {
        const int ch = q >> 5, l = q & 31;
        const int row = a + (ch >> 1) * 4 + (l >> 3), col = 16 * h + (ch & 1) * 8 + (l & 7);
        if (row < b && row < n && col < ncl) Z[row + ldz * (long)(c0 + col)] = ring[(row & (RING - 1)) * Q2R_LD + col];
    }
}

// G groups per round, a ring of RING rows (a power of two >= 2 NB G)
template <int G, int RING>
__global__ void __launch_bounds__(G * 64, 1) q2p_apply_kernel(int n, int S, int ncol,
                                                                 const double *__restrict__ V2,
                                                                 const double *__restrict__ Tq, double *Z,
                                                                 long ldz, int *err)
{
    static_assert(RING >= 2 * NB * G && (RING & (RING - 1)) == 0, "ring size");
    extern __shared__ __align__(16) double q2p_sm[];
    __shared__ volatile int prog[G][2];
    double *ring = q2p_sm;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, lr = lane >> 2, lc = lane & 3;
    const int pr = wid >> 1, h = wid & 1;                        // pair (group slot), half
    double *Vd = q2p_sm + RING * Q2R_LD + pr * Q2P_PAIR;     // V(r, q) at r LD + q, 64 rows
    double *Tsm = Vd + 2 * NB * Q2R_LD;                          // T(q, l) at q + LD l
    double *Wb = Tsm + NB * Q2R_LD;                              // W(q, c) at q LD + c, this half's columns
    const int c0 = blockIdx.x * 32, ncl = min(32, ncol - c0);
    const int ng = (n - 2 + NB - 1) / NB;
    // entries of the dense band outside the parallelogram stay zero; the band is rewritten per block
    for (int e = 32 * h + lane; e < 2 * NB * Q2R_LD; e += 64) Vd[e] = 0.0;
    for (int g0 = ng - 1; g0 >= 0; g0 -= G) {
        const int gl = max(g0 - G + 1, 0), nw = g0 - gl + 1;
        __syncthreads();
        q2r_xfer<RING>(ring, Z, ldz, n, c0, ncl, gl * NB + 1, g0 * NB + 1 + 2 * NB, false, tid, blockDim.x);
        if (tid < 2 * G) prog[tid >> 1][tid & 1] = 0;
        __syncthreads();
        const int ilast = sweep_steps(n, gl * NB);
        if (pr < nw) {
            const int g = g0 - pr;
            const int imax = sweep_steps(n, g * NB);
            const int iprev = pr > 0 ? sweep_steps(n, (g + 1) * NB) : 0;
            // the next block's reflectors and T, and (pair 0) the next step's new rows of Z, are loaded
            // one step ahead into registers so that their latency hides behind the current block
            double vq[NB / 2], tl[NB / 2], zn[16];
            auto fetch_vt = [&](int i) {
                const int nv = q2_nvalid(n, g, i);
                const double *Vblk = V2 + ((long)(g * NB) * S + i) * NB;
                const double *T = Tq + ((long)g * S + i) * NB * NB;
#pragma unroll
                for (int u = 0; u < NB / 2; u++) {
                    const int q = 16 * h + u;
                    vq[u] = q < nv ? __ldg(Vblk + (long)q * S * NB + lane) : 0.0;
                    tl[u] = __ldg(T + lane + NB * q);               // column l = q of T
                }
            };
            if (imax > 0) fetch_vt(0);
            if (pr == 0 && imax > 1) {
                const int t1 = (g + 1) * NB + 1;
                q2p_fetch(zn, Z, ldz, n, c0, ncl, h, t1 + NB, t1 + 2 * NB, lane);
            }
            for (int i = 0; i < imax; i++) {
                const unsigned long long t0 = gtime();
                if (pr > 0) {
                    const int need = min(i + 1, iprev);
                    while (prog[pr - 1][h] < need)
                        if (gtime() - t0 > WAIT_NS) { atomicExch(err, 3); break; }
                } else if (nw > 1) {
                    const int need = min(i + nw - RING / NB + 1, ilast);
                    while (need > 0 && prog[nw - 1][h] < need)
                        if (gtime() - t0 > WAIT_NS) { atomicExch(err, 3); break; }
                }
                __threadfence_block();
                const int top = (g + i) * NB + 1;
                const int nrow = min(2 * NB - 1, n - top);
                if (pr == 0 && i > 0) {
                    q2p_put<RING>(zn, ring, h, top + NB, top + 2 * NB, lane);
                    if (i + 1 < imax) q2p_fetch(zn, Z, ldz, n, c0, ncl, h, top + 2 * NB, top + 3 * NB, lane);
                }
                // ---- the pair stages the block's V band and T (after both finished the previous block) ----
                pair_sync(pr);
                {
                    // compact V(q, t) into the W area first (free until W is formed): consecutive stores
                    double *Vc = Wb;
#pragma unroll
                    for (int u = 0; u < NB / 2; u++) {
                        const int q = 16 * h + u;
                        Vc[q * 33 + lane] = vq[u];
                        Tsm[lane + Q2R_LD * q] = tl[u];
                    }
                    if (i + 1 < imax) fetch_vt(i + 1);
                    pair_sync(pr);
                    // the band V(q + t, q) = Vc(q, t): lane q, 16 values of t per warp (Vc at 33 q + t and
                    // Vd at 37 q + 36 t are distinct banks across a half-warp)
#pragma unroll
                    for (int u = 0; u < NB / 2; u++) {
                        const int t = 16 * h + u, rr = lane + t;
                        Vd[rr * Q2R_LD + lane] = rr < nrow ? Vc[lane * 33 + t] : 0.0;
                    }
                }
                pair_sync(pr);
                // ---- W = V^T Zw on this half's columns: M = q (4), N = column (2), K = row (16) ----
                double acc[4][2][2];
#pragma unroll
                for (int a = 0; a < 4; a++)
#pragma unroll
                    for (int b = 0; b < 2; b++) acc[a][b][0] = acc[a][b][1] = 0.0;
#pragma unroll
                for (int ks = 0; ks < 16; ks++) {
                    const int r = 4 * ks + lc;
                    const double *rrow = ring + ((top + r) & (RING - 1)) * Q2R_LD + 16 * h;
                    const double bz0 = rrow[lr], bz1 = rrow[8 + lr];
#pragma unroll
                    for (int mt = 0; mt < 4; mt++) {
                        if (ks < 2 * mt || ks >= 2 * mt + 10) continue;
                        const double a = Vd[r * Q2R_LD + 8 * mt + lr];
                        q2r_mma(acc[mt][0][0], acc[mt][0][1], a, bz0);
                        q2r_mma(acc[mt][1][0], acc[mt][1][1], a, bz1);
                    }
                }
#pragma unroll
                for (int mt = 0; mt < 4; mt++)
#pragma unroll
                    for (int nt = 0; nt < 2; nt++) {
                        Wb[(8 * mt + lr) * Q2R_LD + 16 * h + 8 * nt + 2 * lc] = acc[mt][nt][0];
                        Wb[(8 * mt + lr) * Q2R_LD + 16 * h + 8 * nt + 2 * lc + 1] = acc[mt][nt][1];
                        acc[mt][nt][0] = acc[mt][nt][1] = 0.0;
                    }
                __syncwarp();
                // ---- W2 = T W ----
#pragma unroll
                for (int ks = 0; ks < 8; ks++) {
                    const int l = 4 * ks + lc;
                    const double bw0 = Wb[l * Q2R_LD + 16 * h + lr], bw1 = Wb[l * Q2R_LD + 16 * h + 8 + lr];
#pragma unroll
                    for (int mt = 0; mt < 4; mt++) {
                        if (ks < 2 * mt) continue;
                        const double a = Tsm[(8 * mt + lr) + Q2R_LD * l];
                        q2r_mma(acc[mt][0][0], acc[mt][0][1], a, bw0);
                        q2r_mma(acc[mt][1][0], acc[mt][1][1], a, bw1);
                    }
                }
                __syncwarp();
#pragma unroll
                for (int mt = 0; mt < 4; mt++)
#pragma unroll
                    for (int nt = 0; nt < 2; nt++) {
                        Wb[(8 * mt + lr) * Q2R_LD + 16 * h + 8 * nt + 2 * lc] = acc[mt][nt][0];
                        Wb[(8 * mt + lr) * Q2R_LD + 16 * h + 8 * nt + 2 * lc + 1] = acc[mt][nt][1];
                    }
                __syncwarp();
                // ---- Zw -= V W2: M = window row (8 tiles in two halves), N = column (2), K = q (8) ----
#pragma unroll
                for (int mh = 0; mh < 2; mh++) {
#pragma unroll
                    for (int a = 0; a < 4; a++) {
                        const int r = 8 * (4 * mh + a) + lr;
                        const double *rrow = ring + ((top + r) & (RING - 1)) * Q2R_LD + 16 * h;
#pragma unroll
                        for (int nt = 0; nt < 2; nt++) {
                            acc[a][nt][0] = rrow[8 * nt + 2 * lc];
                            acc[a][nt][1] = rrow[8 * nt + 2 * lc + 1];
                        }
                    }
#pragma unroll
                    for (int ks = 0; ks < 8; ks++) {
                        const int q = 4 * ks + lc;
                        const double bw0 = Wb[q * Q2R_LD + 16 * h + lr], bw1 = Wb[q * Q2R_LD + 16 * h + 8 + lr];
#pragma unroll
                        for (int a = 0; a < 4; a++) {
                            const int mt = 4 * mh + a;
                            const int klo = 2 * mt - 8 > 0 ? 2 * mt - 8 : 0, khi = 2 * mt + 1 < 7 ? 2 * mt + 1 : 7;
                            if (ks < klo || ks > khi) continue;
                            const double v = -Vd[(8 * mt + lr) * Q2R_LD + q];
                            q2r_mma(acc[a][0][0], acc[a][0][1], v, bw0);
                            q2r_mma(acc[a][1][0], acc[a][1][1], v, bw1);
                        }
                    }
#pragma unroll
                    for (int a = 0; a < 4; a++) {
                        const int r = 8 * (4 * mh + a) + lr;
                        if (r < nrow) {
                            double *rrow = ring + ((top + r) & (RING - 1)) * Q2R_LD + 16 * h;
#pragma unroll
                            for (int nt = 0; nt < 2; nt++) {
                                rrow[8 * nt + 2 * lc] = acc[a][nt][0];
                                rrow[8 * nt + 2 * lc + 1] = acc[a][nt][1];
                            }
                        }
                    }
                }
                __syncwarp();
                if (pr == nw - 1) q2p_store<RING>(ring, Z, ldz, n, c0, ncl, h, top, top + NB, lane);
                __threadfence_block();
                __syncwarp();
                if (lane == 0) prog[pr][h] = i + 1;
            }
        }
        __syncthreads();
        const int rdone = ilast > 0 ? (gl + ilast) * NB + 1 : gl * NB + 1;
        q2r_xfer<RING>(ring, Z, ldz, n, c0, ncl, rdone, n, true, tid, blockDim.x);
    }
}

// ---------------------------------------------------------------------------
// back-transformation of the stage-1 panels, Q1_GROUP panels at a time
// ---------------------------------------------------------------------------
constexpr int Q1_GROUP = 8;
constexpr int Q1W = Q1_GROUP * NB;     // columns of a merged block reflector
constexpr int Q1H = 4 * NB;            // the unit of q1_tmerge_kernel: four panels

struct Q1Panels {
    const double *V[Q1_GROUP];   // V of each panel (m_q x NB, ld m_q), null past the last panel
    int m[Q1_GROUP];
};

// Vg (m0 x Q1W, ld m0): panel q's V shifted down by q NB rows, zeros above
__global__ void q1_gather_kernel(int m0, Q1Panels P, double *Vg)
{
    const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (idx >= (long)m0 * Q1W) return;
    const int r = (int)(idx % m0), c = (int)(idx / m0), q = c / NB, cc = c % NB;
    double v = 0.0;
    if (P.V[q] && r >= q * NB) v = P.V[q][(r - q * NB) + (long)P.m[q] * cc];
    Vg[idx] = v;
}

// The same T from the panels' own T factors (T1) and the Gram blocks, merging pairs as
// Q_a Q_b = I - [V_a V_b] [[T_a, -T_a G_ab T_b], [0, T_b]] [V_a V_b]^T (the block form of the
// recurrence above): two 32 x 32 merges, then one of the 64-column halves; small products in
// shared memory instead of 128 dependent column steps.
constexpr int Q1M_SMEM = (Q1H * (Q1H + 1) + 64 * 65) * (int)sizeof(double);

// T of the merged reflector of four consecutive panels (q0 .. q0+3 of the group): G and the
// output block T are Q1H x Q1H with leading dimension Q1W
__global__ void __launch_bounds__(Q1H) q1_tmerge_kernel(const double *__restrict__ G, Q1Panels P, int q0,
                                                        const double *__restrict__ T1, int p0, double *Tg)
{
    extern __shared__ __align__(16) double q1m_sm[];
    double (*Ts)[Q1H + 1] = (double (*)[Q1H + 1])q1m_sm;               // Ts[r][c]
    double (*W)[65] = (double (*)[65])(q1m_sm + Q1H * (Q1H + 1));
    const int t = threadIdx.x;
    for (int c = 0; c < Q1H; c++) Ts[t][c] = 0.0;
    __syncthreads();
    for (int q = 0; q < 4; q++) {
        if (!P.V[q0 + q]) continue;
        const double *Tp = T1 + (size_t)(p0 + q0 + q) * NB * NB;        // column-major NB x NB
        for (int e = t; e < NB * NB; e += Q1H) Ts[q * NB + e % NB][q * NB + e / NB] = Tp[e];
    }
    __syncthreads();
    // merges: width w = NB (pairs 0|1, 2|3), then 2 NB (halves)
    for (int w = NB; w < Q1H; w *= 2) {
        for (int a0 = 0; a0 < Q1H; a0 += 2 * w) {
            const int b0 = a0 + w;
            for (int e = t; e < w * w; e += Q1H) {
                const int r = e % w, c = e / w;
                double sacc = 0.0;
                for (int k = 0; k <= c; k++) sacc += __ldg(G + (a0 + r) + (long)Q1W * (b0 + k)) * Ts[b0 + k][b0 + c];
                W[r][c] = sacc;
            }
            __syncthreads();
            for (int e = t; e < w * w; e += Q1H) {
                const int r = e % w, c = e / w;
                double sacc = 0.0;
                for (int k = r; k < w; k++) sacc += Ts[a0 + r][a0 + k] * W[k][c];
                Ts[a0 + r][b0 + c] = -sacc;
            }
            __syncthreads();
        }
    }
    for (int c = 0; c < Q1H; c++) Tg[t + (long)Q1W * c] = Ts[t][c];
}

}  // namespace

// ---- stage 1 driver ----
struct Sy2sbWork {
    double *VYV;       // m x 3NB
    double *VYV2;      // the second [V | Y | V] buffer (panels alternate while the look-ahead runs)
    cudaStream_t aux;  // the look-ahead's second stream (null: one stream)
    cudaEvent_t ev_y, ev_c2;
    double *X;         // m x NB
    double *T;         // NB x NB
    double *Mp;        // chunks x NB x NB
    double *part;      // PQ CTAs x 4NB
    double *gram;      // PQ CTAs x NB x NB
    unsigned *bar;     // 2
    unsigned *ticket;  // ypass1's last-CTA counter (zero between panels)
    int *err;
    double *gemm_ws;   // split-K workspace
    size_t gemm_ws_doubles;
};

int sy2sb_panels(int n) { return n > NB ? (n - 1) / NB : 0; }   // panels j = 0, NB, ... with j + NB < n

// Saved panels for the back-transformation: V of panel p (m_p x NB, ld m_p) at Vsave + voff(p),
// T of panel p at Tsave + p NB^2.
size_t sy2sb_vsave_doubles(int n)
{
    size_t t = 0;
    for (int j = 0; j + NB < n; j += NB) t += (size_t)(n - j - NB) * NB;
    return t + 64;
}

int sy2sb(cudaStream_t st, int n, double *A, long lda, double *Vsave, double *Tsave, const Sy2sbWork &w)
{
    cudaError_t e;
    const int smem = PQ_ROWS * (NB + 1) * (int)sizeof(double);
    if ((e = smem_attr(panel_qr_kernel, smem)) != cudaSuccess ||
        (e = smem_attr(ypass1_kernel, YP1_SMEM)) != cudaSuccess)
        return cuda_fail(e, "sy2sb smem");
    // the cluster form of the panel factorisation when a 16-CTA cluster with its shared memory fits
    // (BSRG_PANEL_GRID selects the grid-barrier form)
    bool use_cluster = !getenv("BSRG_PANEL_GRID");
    if (use_cluster) {
        const int smem_c = (PQC_ROWS * (NB + 1) + 4 * NB + NB * NB) * (int)sizeof(double);
        if (cudaFuncSetAttribute(panel_qr_cluster_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
                cudaSuccess ||
            smem_attr(panel_qr_cluster_kernel, smem_c) !=
                cudaSuccess) {
            use_cluster = false;
        } else {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(PQC_MAXG);
            cfg.blockDim = dim3(PQ_NT);
            cfg.dynamicSmemBytes = (size_t)smem_c;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = PQC_MAXG;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            int nclusters = 0;
            if (cudaOccupancyMaxActiveClusters(&nclusters, panel_qr_cluster_kernel, &cfg) != cudaSuccess ||
                nclusters < 1)
                use_cluster = false;
        }
        cudaGetLastError();
    }
    // factorise panel p (columns j = p NB ..) on stream sq; its V goes to the [V | Y | V] buffer of p's parity
    auto factor_panel = [&](int p, size_t voff, cudaStream_t sq) -> int {
        const int j = p * NB, m = n - j - NB;
        int G = (m + PQ_ROWS - 1) / PQ_ROWS;
        G = std::max(1, std::min(G, std::max(1, m / NB)));      // CTA 0 holds the NB pivot rows
        const int rpc = (m + G - 1) / G;
        if (rpc > PQ_ROWS) { set_error("sy2sb: panel of %d rows does not fit", m); return BSRG_ERR_ARG; }
        PanelArgs a;
        a.P = A + (j + NB) + lda * (long)j;
        a.ldp = lda;
        a.m = m;
        a.rpc = rpc;
        a.V = (p & 1) && w.aux ? w.VYV2 : w.VYV;
        a.Vs = Vsave + voff;
        a.T = w.T;
        a.Ts = Tsave + (size_t)p * NB * NB;
        a.part = w.part;
        a.gram = w.gram;
        a.bar = w.bar;
        a.err = w.err;
        const int Gc = std::max(1, (m + PQC_ROWS - 1) / PQC_ROWS);
        if (use_cluster && Gc <= PQC_MAXG) {
            // one cluster of Gc CTAs (m / Gc rows each)
            a.rpc = (m + Gc - 1) / Gc;
            const int smem_c = (a.rpc * (NB + 1) + 4 * NB + NB * NB) * (int)sizeof(double);
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3((unsigned)Gc);
            cfg.blockDim = dim3(PQ_NT);
            cfg.dynamicSmemBytes = (size_t)smem_c;
            cfg.stream = sq;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = (unsigned)Gc;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            if ((e = cudaLaunchKernelEx(&cfg, panel_qr_cluster_kernel, a)) != cudaSuccess)
                return cuda_fail(e, "sy2sb panel (cluster)");
        } else {
            void *args[] = {&a};
            if ((e = cudaLaunchCooperativeKernel((const void *)panel_qr_kernel, G, PQ_NT, args, smem, sq)) !=
                cudaSuccess)
                return cuda_fail(e, "sy2sb panel");
        }
        return BSRG_OK;
    };
    size_t voff = 0;
    int rc = n > NB ? factor_panel(0, 0, st) : BSRG_OK;
    if (rc != BSRG_OK) return rc;
    bool qr_on_aux = false;                       // the current panel was factorised on the aux stream
    int p = 0;
    for (int j = 0; j + NB < n; j += NB, p++) {
        const int m = n - j - NB;
        double *VYV = (p & 1) && w.aux ? w.VYV2 : w.VYV;
        double *A22 = A + (j + NB) + lda * (long)(j + NB);
        double *Vp = VYV, *Yp = VYV + (long)m * NB;
        const size_t voff_next = voff + (size_t)m * NB;
        const bool has_next = j + 2 * NB < n;
        if (qr_on_aux && (e = cudaStreamWaitEvent(st, w.ev_c2, 0)) != cudaSuccess)
            return cuda_fail(e, "sy2sb look-ahead wait");
        // X = A22 V with A22 read from its lower triangle (only the lower triangle is updated)
        DgemmBatch gx{};
        gx.m = m; gx.n = NB; gx.k = m;
        gx.A = A22; gx.lda = lda; gx.B = Vp; gx.ldb = m; gx.C = w.X; gx.ldc = m;
        gx.alpha = 1.0; gx.beta = 0.0; gx.syma = 1;
        rc = dgemm_ws(false, false, gx, 1, st, w.gemm_ws, w.gemm_ws_doubles);
        if (rc != BSRG_OK) return rc;
        const int nch = (m + 127) / 128;
        ypass1_kernel<<<nch, 128, YP1_SMEM, st>>>(m, w.X, Vp, w.T, Yp, w.Mp, w.ticket);
        ypass2_kernel<<<nch, 128, 0, st>>>(m, Vp, w.Mp + (size_t)nch * NB * NB, Yp);
        // A22 -= [V Y] [Y V]^T, the tiles that reach the lower triangle
        if (!w.aux || m <= NB) {
            DgemmBatch gu{};
            gu.m = m; gu.n = m; gu.k = 2 * NB;
            gu.A = VYV; gu.lda = m; gu.B = Yp; gu.ldb = m; gu.C = A22; gu.ldc = lda;
            gu.alpha = -1.0; gu.beta = 1.0; gu.lowc = 1;
            rc = dgemm_ws(false, true, gu, 1, st, nullptr, 0);
            if (rc == BSRG_OK && has_next) rc = factor_panel(p + 1, voff_next, st);
            if (rc != BSRG_OK) return rc;
            qr_on_aux = false;
        } else {
            // look-ahead: the next panel's NB columns first; the next panel is then factorised on the
            // high-priority aux stream while the rest of the trailing matrix is updated here, so the
            // panel's few CTAs are placed before the update's fill the machine
            DgemmBatch g1{};
            g1.m = m; g1.n = NB; g1.k = 2 * NB;
            g1.A = VYV; g1.lda = m; g1.B = Yp; g1.ldb = m; g1.C = A22; g1.ldc = lda;
            g1.alpha = -1.0; g1.beta = 1.0;
            rc = dgemm_ws(false, true, g1, 1, st, nullptr, 0);
            if (rc != BSRG_OK) return rc;
            qr_on_aux = false;
            if (has_next) {
                if ((e = cudaEventRecord(w.ev_y, st)) != cudaSuccess ||
                    (e = cudaStreamWaitEvent(w.aux, w.ev_y, 0)) != cudaSuccess)
                    return cuda_fail(e, "sy2sb look-ahead");
                rc = factor_panel(p + 1, voff_next, w.aux);
                if (rc != BSRG_OK) return rc;
                if ((e = cudaEventRecord(w.ev_c2, w.aux)) != cudaSuccess) return cuda_fail(e, "sy2sb look-ahead");
                qr_on_aux = true;
            }
            const int m2 = m - NB;
            DgemmBatch g2{};
            g2.m = m2; g2.n = m2; g2.k = 2 * NB;
            g2.A = VYV + NB; g2.lda = m; g2.B = Yp + NB; g2.ldb = m; g2.C = A22 + NB + lda * (long)NB; g2.ldc = lda;
            g2.alpha = -1.0; g2.beta = 1.0; g2.lowc = 1;
            rc = dgemm_ws(false, true, g2, 1, st, nullptr, 0);
            if (rc != BSRG_OK) return rc;
        }
        voff = voff_next;
    }
    if (qr_on_aux && (e = cudaStreamWaitEvent(st, w.ev_c2, 0)) != cudaSuccess)
        return cuda_fail(e, "sy2sb look-ahead join");
    return cuda_fail(cudaGetLastError(), "sy2sb");
}

}  // namespace bsrg

namespace bsrg {

int symmetrize_lower(int n, const double *A, long lda, double *F, long ldf, cudaStream_t s);   // refine.cu

// Workspace of dense_syevd in doubles (everything but the output Z)
// The workspace carve-up of syevd2_impl, as offsets (doubles, 32-aligned); the size
// function and the solver use this one layout.
struct Syevd2Layout {
    size_t Wk, AB, V1, T1, V2, tau2, Tq, dv, ev, progress, VYV, X, T, Mp, part, gram, flags, W1, W2, Vg, Gq, Tg,
        gemm_ws, dcw, total;
};

static Syevd2Layout syevd2_layout(int n)
{
    Syevd2Layout L{};
    const size_t nn = (size_t)n * n;
    const size_t S = (size_t)sweep_steps(n, 0) + 1, ng = (size_t)(n + NB - 1) / NB + 1;
    size_t off = 0;
    auto take = [&](size_t cnt) { off = (off + 31) & ~(size_t)31; size_t p = off; off += cnt; return p; };
    L.Wk = take(nn);
    L.AB = take((size_t)LDAB * n);
    L.V1 = take(sy2sb_vsave_doubles(n));
    L.T1 = take((size_t)(sy2sb_panels(n) + 1) * NB * NB);
    L.V2 = take((size_t)n * S * NB);
    L.tau2 = take((size_t)n * S);
    L.Tq = take(ng * S * NB * NB);
    L.dv = take(n);
    L.ev = take(n + 1);
    L.progress = take(n / 2 + 8);
    L.VYV = take((size_t)n * 6 * NB);               // two [V | Y | V] buffers
    L.X = take((size_t)n * NB);
    L.T = take(NB * NB);
    L.Mp = take(((size_t)n / 128 + 2) * NB * NB);
    L.part = take((size_t)(n / NB + 8) * 4 * NB);
    L.gram = take((size_t)(n / NB + 8) * NB * NB);
    L.flags = take(8);
    L.W1 = take((size_t)Q1W * n);
    L.W2 = take(std::max((size_t)Q1W * n, (size_t)(Q1W / 2) * (Q1W / 2)));   // also the T merges' temporary
    L.Vg = take((size_t)Q1W * n);
    L.Gq = take((size_t)Q1W * Q1W);
    L.Tg = take((size_t)Q1W * Q1W);
    L.gemm_ws = take(8 * (size_t)Q1W * n);
    L.dcw = take(dc_workspace_bytes(n) / 8 + 8);
    L.total = off + 64;
    return L;
}

size_t syevd2_workspace_doubles(int n) { return syevd2_layout(n).total; }

// Eigenvalues (ascending, w) and eigenvectors (Z, ldz) of the symmetric A (lower
// triangle referenced).  Z may be A itself.  ws: syevd2_workspace_doubles(n).
// tri_d / tri_e non-null: stop after the reduction and copy the tridiagonal (d: n, e: n-1) there
static int syevd2_impl(bsrg_ctx *c, int n, const double *A, long lda, double *w, double *Z, long ldz, double *ws,
                       size_t ws_doubles, void *pinned, size_t pinned_bytes, int *launches, double *tri_d,
                       double *tri_e)
{
    int nl = 0;
    if (n < 1) return BSRG_OK;
    cudaStream_t st = c->stream;
    cudaError_t e;
    if (ws_doubles < syevd2_workspace_doubles(n)) { set_error("dsyevd: workspace too small"); return BSRG_ERR_NOMEM; }
    if (n > 10240) { set_error("dsyevd: n=%d above 10240", n); return BSRG_ERR_ARG; }
    const int S = sweep_steps(n, 0) + 1;
    const Syevd2Layout L = syevd2_layout(n);
    double *Wk = ws + L.Wk, *AB = ws + L.AB, *V1 = ws + L.V1, *T1 = ws + L.T1;
    double *V2 = ws + L.V2, *tau2 = ws + L.tau2, *Tq = ws + L.Tq;
    double *dv = ws + L.dv, *ev = ws + L.ev;
    int *progress = (int *)(ws + L.progress);
    Sy2sbWork sw;
    sw.VYV = ws + L.VYV;
    sw.VYV2 = sw.VYV + (size_t)n * 3 * NB;
    sw.aux = getenv("BSRG_NO_LOOKAHEAD") ? nullptr : c->aux_stream;
    sw.ev_y = c->aux_ev[0];
    sw.ev_c2 = c->aux_ev[1];
    sw.X = ws + L.X;
    sw.T = ws + L.T;
    sw.Mp = ws + L.Mp;
    sw.part = ws + L.part;
    sw.gram = ws + L.gram;
    int *flags = (int *)(ws + L.flags);            // bar[2], err, err2
    sw.bar = (unsigned *)flags;
    sw.err = flags + 2;
    sw.ticket = (unsigned *)(flags + 4);
    double *W1 = ws + L.W1, *W2 = ws + L.W2;
    double *Vg = ws + L.Vg, *Gq = ws + L.Gq, *Tg = ws + L.Tg;
    sw.gemm_ws_doubles = 8 * (size_t)Q1W * n;
    sw.gemm_ws = ws + L.gemm_ws;
    double *dcw = ws + L.dcw;
    if ((e = cudaMemsetAsync(flags, 0, 8 * sizeof(int), st)) != cudaSuccess ||
        (e = cudaMemsetAsync(progress, 0, sizeof(int) * n, st)) != cudaSuccess)
        return cuda_fail(e, "dsyevd init");
    const int np = sy2sb_panels(n);
    double fl_band = 0.0, fl_chase = 0.0, fl_q2 = 0.0, fl_q1 = 0.0, fl_dc = 0.0;
    for (int j = 0; j + NB < n; j += NB) {
        const double m = n - j - NB;
        // X (2 m^2 NB), the lower-triangle tiles of the rank-2NB update (~2 m^2 NB), QR and Y passes
        fl_band += 4.0 * m * m * NB + 6.0 * m * NB * NB + 4.0 * m * NB * NB;
        fl_q1 += 4.0 * (m + 1.5 * NB) * n * NB + 2.0 * Q1W * NB * n + 2.0 * Q1W * NB * m;  // per panel share of a group
    }
    // 1. full symmetric working copy, dense -> band
    stage_begin(c, 9);
    int rc = symmetrize_lower(n, A, lda, Wk, n, st);
    if (rc == BSRG_OK) rc = sy2sb(st, n, Wk, n, V1, T1, sw);
    if (rc != BSRG_OK) return rc;
    band_extract_kernel<<<(unsigned)(((long)n * LDAB + 255) / 256), 256, 0, st>>>(n, Wk, n, AB);
    stage_end(c, 9, 2 + np * 6);
    c->stage_flops[9] += fl_band;
    stage_begin(c, 10);
    // 2. band -> tridiagonal
    if (n > 2) {
        int nsm = 148;
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
        // the register form with a helper warp (sb2st3_kernel) by default; BSRG_SB2ST_ONEWARP selects the
        // register form without it, groups of SB_K consecutive sweeps per CTA (sb2st2_kernel<SB_K>), and
        // BSRG_SB2ST_SHARED the shared-memory form with one sweep per CTA
        constexpr int SB_K = 1;              // eight sweeps per CTA measured slower (152 vs 121 ms at n = 7810)
        Sb2stArgs a2{AB, n, V2, tau2, S, progress, sw.err};
        void *args[] = {&a2};
        if (!getenv("BSRG_SB2ST_SHARED") && !getenv("BSRG_SB2ST_ONEWARP")) {
            // one sweep per CTA at a time: the chain of reflectors and right updates on one warp, the
            // diagonal blocks and the left updates on two more, a helper warp that publishes the steps
            // (sb2st5_kernel; BSRG_SB2ST_TWOWARP: sb2st3_kernel, computing warp and helper only).  A sweep
            // starts three steps behind its predecessor, so about sweep_steps / 3 sweeps are active at
            // once; sweep_steps / 2.5 + 4 CTAs (at most one per SM) never make a sweep wait for its CTA,
            // and the SMs left over stay free for work on other streams instead of polling
            // (BSRG_SB2ST_CTAS overrides the count)
            int want = (int)(sweep_steps(n, 0) / 2.5) + 4;
            if (const char *ov = getenv("BSRG_SB2ST_CTAS")) want = std::max(1, atoi(ov));
            const int ctas = std::max(1, std::min(n - 2, std::min(nsm, want)));
            const bool two = getenv("BSRG_SB2ST_TWOWARP") != nullptr;
            if ((e = cudaLaunchCooperativeKernel(two ? (const void *)sb2st3_kernel : (const void *)sb2st5_kernel, ctas,
                                                 two ? 64 : 128, args, 0, st)) != cudaSuccess)
                return cuda_fail(e, "dsyevd bulge chasing");
        } else if (getenv("BSRG_SB2ST_SHARED")) {
            int per = 1;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, sb2st_kernel, 32, 0);
            const int workers = std::max(1, std::min(n - 2, std::min(nsm * std::max(per, 1), 2 * nsm)));
            if ((e = cudaLaunchCooperativeKernel((const void *)sb2st_kernel, workers, 32, args, 0, st)) != cudaSuccess)
                return cuda_fail(e, "dsyevd bulge chasing");
        } else {
            const int smem = SB_K * SB_WSM * (int)sizeof(double);
            if ((e = smem_attr(sb2st2_kernel<SB_K>, smem)) !=
                cudaSuccess)
                return cuda_fail(e, "dsyevd bulge chasing smem");
            int per = 1;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, sb2st2_kernel<SB_K>, 32 * SB_K, smem);
            const int groups = (n - 2 + SB_K - 1) / SB_K;
            const int ctas = std::max(1, std::min(groups, std::min(nsm * std::max(per, 1), 2 * nsm)));
            if ((e = cudaLaunchCooperativeKernel((const void *)sb2st2_kernel<SB_K>, ctas, 32 * SB_K, args, smem, st)) !=
                cudaSuccess)
                return cuda_fail(e, "dsyevd bulge chasing");
        }
    }
    tridiag_extract_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, AB, dv, ev);
    for (int j = 0; j < n - 2; j++)
        for (int i = 0; i < sweep_steps(n, j); i++) {
            const double L = std::min(NB, n - (j + 1 + i * NB)), nlf = i == 0 ? 0 : NB - 1;
            const double nb2 = std::max(0, std::min(NB, n - (j + 1 + i * NB) - (int)L));
            fl_chase += 4.0 * L * (nlf + L + nb2);
        }
    stage_end(c, 10, 2);
    c->stage_flops[10] += fl_chase;
    if (tri_d) {
        int hf = 0;
        if ((e = cudaMemcpyAsync(tri_d, dv, sizeof(double) * n, cudaMemcpyDeviceToDevice, st)) != cudaSuccess ||
            (n > 1 && (e = cudaMemcpyAsync(tri_e, ev, sizeof(double) * (n - 1), cudaMemcpyDeviceToDevice, st)) !=
                          cudaSuccess) ||
            (e = cudaMemcpyAsync(&hf, flags + 2, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (e = cudaStreamSynchronize(st)) != cudaSuccess)
            return cuda_fail(e, "dsytrd_2stage");
        if (hf != 0) {
            set_error("dsytrd_2stage: a device-side wait timed out (%s)", hf == 2 ? "bulge chasing" : "panel barrier");
            return BSRG_ERR_CUDA;
        }
        return BSRG_OK;
    }
    // 3. tridiagonal eigenpairs into Z
    stage_begin(c, 11);
    int ndc = 0;
    rc = tridiag_dc(st, n, dv, ev, w, Z, ldz, dcw, dc_workspace_bytes(n), pinned, pinned_bytes, &fl_dc, &ndc);
    if (rc != BSRG_OK) return rc;
    stage_end(c, 11, ndc);
    c->stage_flops[11] += fl_dc;
    // 4. back-transformation: Q2 then Q1
    stage_begin(c, 12);
    if (n > 2) {
        dim3 gt((unsigned)S, (unsigned)((n - 2 + NB - 1) / NB));
        q2_tfactor_kernel<<<gt, 32, 0, st>>>(n, S, V2, tau2, Tq);
        if ((e = smem_attr(q2_apply_kernel, Q2_SMEM)) !=
            cudaSuccess)
            return cuda_fail(e, "dsyevd Q2 smem");
        if (getenv("BSRG_Q2_SIMPLE")) {
            q2_apply_kernel<<<(unsigned)((n + Q2_COLS - 1) / Q2_COLS), Q2_NT, Q2_SMEM, st>>>(n, S, n, V2, Tq, Z, ldz);
        } else if (getenv("BSRG_Q2_WAVE")) {
            if ((e = smem_attr(q2w_apply_kernel, Q2W_SMEM)) !=
                cudaSuccess)
                return cuda_fail(e, "dsyevd Q2 smem");
            q2w_apply_kernel<<<(unsigned)((n + 31) / 32), Q2W_WARPS * 32, Q2W_SMEM, st>>>(n, S, n, V2, Tq, Z, ldz,
                                                                                          sw.err);
        } else if (getenv("BSRG_Q2_RING1")) {
            if ((e = smem_attr(q2r_apply_kernel, Q2R_SMEM)) !=
                cudaSuccess)
                return cuda_fail(e, "dsyevd Q2 smem");
            q2r_apply_kernel<<<(unsigned)((n + 31) / 32), Q2R_W * 32, Q2R_SMEM, st>>>(n, S, n, V2, Tq, Z, ldz, sw.err);
        } else {
            // four groups per round and one CTA per SM, or (BSRG_Q2_TWO) two groups and two CTAs per SM
            if (getenv("BSRG_Q2_TWO")) {
                constexpr int sm2 = q2p_smem<2, 128>();
                if ((e = smem_attr(q2p_apply_kernel<2, 128>, sm2)) != cudaSuccess)
                    return cuda_fail(e, "dsyevd Q2 smem");
                q2p_apply_kernel<2, 128><<<(unsigned)((n + 31) / 32), 2 * 64, sm2, st>>>(n, S, n, V2, Tq, Z, ldz,
                                                                                        sw.err);
            } else {
                constexpr int sm4 = q2p_smem<4, 256>();
                if ((e = smem_attr(q2p_apply_kernel<4, 256>, sm4)) != cudaSuccess)
                    return cuda_fail(e, "dsyevd Q2 smem");
                q2p_apply_kernel<4, 256><<<(unsigned)((n + 31) / 32), 4 * 64, sm4, st>>>(n, S, n, V2, Tq, Z, ldz,
                                                                                        sw.err);
            }
        }
        // per block and column: W = V^T Z (2 NB nv), T W (~NB nv), Z -= V W (2 NB nv)
        double nvsum = 0.0;
        for (int j = 0; j < n - 2; j++) nvsum += sweep_steps(n, j);
        fl_q2 = 5.0 * NB * nvsum * n;
    }
    stage_end(c, 12, n > 2 ? 2 : 0);
    c->stage_flops[12] += fl_q2;
    stage_begin(c, 13);
    {
        std::vector<size_t> voff;
        size_t vo = 0;
        for (int j = 0; j + NB < n; j += NB) { voff.push_back(vo); vo += (size_t)(n - j - NB) * NB; }
        const int ngrp = (np + Q1_GROUP - 1) / Q1_GROUP;
        for (int gq = ngrp - 1; gq >= 0; gq--) {
            const int p0 = gq * Q1_GROUP, r0 = p0 * NB + NB, m0 = n - r0;
            Q1Panels P{};
            for (int q = 0; q < Q1_GROUP; q++) {
                const int p = p0 + q;
                P.V[q] = p < np ? V1 + voff[p] : nullptr;
                P.m[q] = p < np ? n - p * NB - NB : 0;
            }
            q1_gather_kernel<<<(unsigned)(((long)m0 * Q1W + 255) / 256), 256, 0, st>>>(m0, P, Vg);
            rc = dgemm(true, false, Q1W, Q1W, m0, 1.0, Vg, m0, Vg, m0, 0.0, Gq, Q1W, st, sw.gemm_ws,
                       sw.gemm_ws_doubles);
            if (rc != BSRG_OK) return rc;
            // T of the merged 256-column reflector: each 128-column half by pairwise merges of its
            // panels' T (q1_tmerge_kernel), then the off-diagonal block -T_a G_ab T_b by two GEMMs
            if ((e = smem_attr(q1_tmerge_kernel, Q1M_SMEM)) != cudaSuccess)
                return cuda_fail(e, "dsyevd Q1 smem");
            if ((e = cudaMemsetAsync(Tg, 0, sizeof(double) * Q1W * Q1W, st)) != cudaSuccess)
                return cuda_fail(e, "dsyevd Q1 T");
            for (int hq = 0; hq < Q1_GROUP / 4; hq++) {
                const long o = (long)hq * Q1H * (Q1W + 1);
                q1_tmerge_kernel<<<1, Q1H, Q1M_SMEM, st>>>(Gq + o, P, 4 * hq, T1, p0, Tg + o);
            }
            for (int w = Q1H; w < Q1W; w *= 2)
                for (int a0 = 0; a0 < Q1W; a0 += 2 * w) {
                    const int b0 = a0 + w;
                    // Wq = G(a, b) T_b (w x w), then T(a, b) = -T_a Wq
                    rc = dgemm(false, false, w, w, w, 1.0, Gq + a0 + (long)Q1W * b0, Q1W, Tg + b0 + (long)Q1W * b0,
                               Q1W, 0.0, W2, w, st);
                    if (rc == BSRG_OK)
                        rc = dgemm(false, false, w, w, w, -1.0, Tg + a0 + (long)Q1W * a0, Q1W, W2, w, 0.0,
                                   Tg + a0 + (long)Q1W * b0, Q1W, st);
                    if (rc != BSRG_OK) return rc;
                }
            double *Zs = Z + r0;
            rc = dgemm(true, false, Q1W, n, m0, 1.0, Vg, m0, Zs, ldz, 0.0, W1, Q1W, st, sw.gemm_ws,
                       sw.gemm_ws_doubles);
            if (rc == BSRG_OK) rc = dgemm(false, false, Q1W, n, Q1W, 1.0, Tg, Q1W, W1, Q1W, 0.0, W2, Q1W, st);
            if (rc == BSRG_OK) rc = dgemm(false, false, m0, n, Q1W, -1.0, Vg, m0, W2, Q1W, 1.0, Zs, ldz, st);
            if (rc != BSRG_OK) return rc;
        }
    }
    stage_end(c, 13, 10 * ((np + Q1_GROUP - 1) / Q1_GROUP));
    c->stage_flops[13] += fl_q1;
    c->stage_flops[6] += fl_band + fl_chase + fl_dc + fl_q2 + fl_q1;
    // device-side waits report through the flags
    int hflag[2] = {0, 0};
    if ((e = cudaMemcpyAsync(hflag, flags + 2, sizeof(int) * 2, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return cuda_fail(e, "dsyevd");
    if (hflag[0] != 0) {
        set_error("dsyevd: a device-side wait timed out (%s)",
                  hflag[0] == 2 ? "bulge chasing" : hflag[0] == 3 ? "back-transformation wavefront" : "panel barrier");
        return BSRG_ERR_CUDA;
    }
    // kernels of this library per call
    nl = 2 + np * 6 + 2 + ndc + (n > 2 ? 2 : 0) + 3 * np;
    if (launches) *launches = nl;
    return BSRG_OK;
}

int dense_syevd(bsrg_ctx *c, int n, const double *A, long lda, double *w, double *Z, long ldz, double *ws,
                size_t ws_doubles, void *pinned, size_t pinned_bytes, int *launches)
{
    return syevd2_impl(c, n, A, lda, w, Z, ldz, ws, ws_doubles, pinned, pinned_bytes, launches, nullptr, nullptr);
}

}  // namespace bsrg

using namespace bsrg;

extern "C" int bsrg_dsytrd_2stage(bsrg_ctx *c, int n, const double *A, int lda, double *d, double *e)
{
    if (!c || (n > 0 && (!A || !d || (n > 1 && !e)))) { set_error("dsytrd_2stage: null argument"); return BSRG_ERR_ARG; }
    if (n < 0 || lda < (n > 0 ? n : 1)) { set_error("dsytrd_2stage: n=%d lda=%d", n, lda); return BSRG_ERR_ARG; }
    if (n == 0) return BSRG_OK;
    cudaSetDevice(c->device);
    int rc = ctx_reserve(c, syevd2_workspace_doubles(n) * sizeof(double) + 1024);
    if (rc != BSRG_OK) return rc;
    rc = syevd2_impl(c, n, A, lda, nullptr, nullptr, n, (double *)c->ws, c->ws_bytes / sizeof(double), nullptr, 0,
                     nullptr, d, e);
    cudaEventRecord(c->ev_stage, c->stream);
    return rc;
}

extern "C" int bsrg_dsyevd(bsrg_ctx *c, int n, const double *A, int lda, double *w, double *Z, int ldz)
{
    if (!c || (n > 0 && (!A || !w || !Z))) { set_error("dsyevd: null argument"); return BSRG_ERR_ARG; }
    if (n < 0 || lda < (n > 0 ? n : 1) || ldz < (n > 0 ? n : 1)) {
        set_error("dsyevd: n=%d lda=%d ldz=%d", n, lda, ldz);
        return BSRG_ERR_ARG;
    }
    if (n == 0) return BSRG_OK;
    cudaSetDevice(c->device);
    int rc = ctx_reserve(c, syevd2_workspace_doubles(n) * sizeof(double) + 1024);
    if (rc == BSRG_OK) rc = ctx_reserve_pinned(c, dc_pinned_bytes(n));
    if (rc != BSRG_OK) return rc;
    rc = dense_syevd(c, n, A, lda, w, Z, ldz, (double *)c->ws, c->ws_bytes / sizeof(double), c->pinned,
                     c->pinned_bytes, nullptr);
    cudaEventRecord(c->ev_stage, c->stream);
    return rc;
}
