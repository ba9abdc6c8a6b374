// Channel-block assembly of one partial wave on the GPU (the bsr_mat hot path).
//
// Reference (src/bsr/BSR_MAT3): SUB1 (sub1.f90:72-191) drives, per partial wave,
//   L_data Case(6..9) (L_data.f90:131-150) with hl_core from INT_core
//   (l_core.f90:174-270): H_ii += -1/2 hl_l  (no closed shells),
//   I_data Case(6..9) (I_data.f90:192-218): for each coefficient group of one
//   channel pair, multipole k and structure, xx = sum_t c_t density(p_a,p_b),
//   dd = convol(xx) and UPDATE_HX (mod_intmat.f90:69) into the block,
//   UPDATE_CF (mod_intmat.f90:245) for the asymptotic coefficients,
//   UPDATE_HL(i,i,sb,Etarg) (sub1.f90:178) and the symmetrisation of the
//   diagonal blocks (sub1.f90:187-191).
//
// B200 layout of the work, per multipole k (all on one stream):
//   rk moments -> rkb_k (ns,ns,ks,ks) in HBM (32 MB at ns=200, ks=10, stays in L2)
//   direct groups:   Xd_g = sum_t c_t density_s(p_a,p_b)          (band (ns,ks))
//                    Out[g,(i,ip)] = sum_(j,jp) Xd_g(j,jp) rkb(i,j,ip,jp)
//                    a register-tiled FP64 GEMM (groups x (ns ks) x (ns ks)) whose
//                    epilogue is UPDATE_HX 's' into the channel block
//   exchange groups: the group density D_g = sum_t c_t p_a p_b^T is built in
//                    shared memory tile by tile (never written to HBM) and the
//                    convol icase-3 gather runs on it for several groups at once,
//                    so every rkb value read from L2 feeds all of them; the
//                    epilogue is UPDATE_HX 'x'.
// A block receives at most one group per (k, structure), so no two CTAs of one
// launch update the same H element and no atomics are needed.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "ctx.h"
#include "dgemm.h"
#include "dmma.cuh"

namespace bsrg {

// ---------------------------------------------------------------------------
// one-electron blocks: hcc_ii = -1/2 * hl_core(l_i)  (hcc zeroed beforehand)
// hl = db2 - l(l+1) rm2 + 2z rm1 with the Bloch fix of INT_core at (ns, ks-1/ks)
// ---------------------------------------------------------------------------
__global__ void one_electron_kernel(int ns, int ks, int nch, const int *__restrict__ lch, double z,
                                    const double *__restrict__ db2, const double *__restrict__ rm2,
                                    const double *__restrict__ rm1, double *hcc)
{
    int ich = blockIdx.y;
    int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= ns * ks || ich >= nch) return;
    int i = tid % ns, jp = tid / ns;            // band (i, jp): element (i, j = i + jp - (ks-1))
    int j = i + jp - (ks - 1);
    if (j < 0) return;
    int l = lch[ich];
    double c1 = (double)(l * (l + 1)), c2 = 2 * z;
    double v = db2[tid] - c1 * rm2[tid] + c2 * rm1[tid];
    if (i == ns - 1 && (jp == ks - 2 || jp == ks - 1)) {
        double cb = db2[0] - db2[(ns - 1) + (size_t)ns * (ks - 2)];
        v = jp == ks - 2 ? v + cb : v - cb;
    }
    double *blk = hcc + ((size_t)(ich + 1) * (ich + 2) / 2 - 1) * ns * ns;
    double x = -0.5 * v;
    blk[i + (size_t)ns * j] += x;
    if (i != j) blk[j + (size_t)ns * i] += x;
}

// UPDATE_HL(ich,ich,sb,c_ich) for all channels; optionally also writes S blocks.
__global__ void sb_update_kernel(int ns, int ks, int nch, const double *__restrict__ ech,
                                 const double *__restrict__ sb, double *hcc, double *scc)
{
    int ich = blockIdx.y;
    int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= ns * ks || ich >= nch) return;
    int i = tid % ns, ith = tid / ns;
    int j = i + ith - (ks - 1);
    if (j < 0) return;
    size_t off = ((size_t)(ich + 1) * (ich + 2) / 2 - 1) * ns * ns;
    double s = sb[tid];
    if (hcc) {
        double v = ech[ich] * s;
        hcc[off + i + (size_t)ns * j] += v;
        if (i != j) hcc[off + j + (size_t)ns * i] += v;
    }
    if (scc) {
        scc[off + i + (size_t)ns * j] = s;
        if (i != j) scc[off + j + (size_t)ns * i] = s;
    }
}

__global__ void symmetrize_diag_kernel(int ns, int nch, double *hcc)
{
    int ich = blockIdx.y;
    int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= ns * ns || ich >= nch) return;
    int i = tid % ns, j = tid / ns;
    if (j > i) return;
    double *blk = hcc + ((size_t)(ich + 1) * (ich + 2) / 2 - 1) * ns * ns;
    double c = blk[i + (size_t)ns * j] + blk[j + (size_t)ns * i];
    blk[i + (size_t)ns * j] = c / 2.0;
    blk[j + (size_t)ns * i] = c / 2.0;
}

// ---------------------------------------------------------------------------
// direct groups
// ---------------------------------------------------------------------------
struct GroupDesc {
    int start, end;   // coefficient range
    int blk;          // 0-based block index i(i-1)/2 + j - 1
    int ich, jch;     // 1-based channels
};

// Xd_g(j,jp) = sum_t c_t * density_s(p_a,p_b)(j,jp)   (I_data.f90:198-199)
__global__ void direct_density_kernel(int ns, int ks, int ng, const GroupDesc *__restrict__ gd,
                                      const int *__restrict__ ca, const int *__restrict__ cb,
                                      const double *__restrict__ cv, const double *__restrict__ P,
                                      double *__restrict__ Xd)
{
    int g = blockIdx.y;
    int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ng || tid >= ns * ks) return;
    int i = tid % ns, jp = tid / ns;
    GroupDesc G = gd[g];
    double acc = 0.0;
    if (i + jp < ns) {
        for (int t = G.start; t < G.end; t++) {
            const double *pa = P + (size_t)ns * ca[t], *pb = P + (size_t)ns * cb[t];
            double dd = jp == 0 ? pa[i] * pb[i] : pa[i] * pb[i + jp] + pa[i + jp] * pb[i];
            acc = fma(cv[t], dd, acc);
        }
    }
    Xd[(size_t)g * ns * ks + tid] = acc;
}

constexpr int XTX = 32;                  // exchange tile rows (lanes)
constexpr int XTYT = 5;                  // exchange columns per thread
constexpr int XTY = 8 * XTYT;            // exchange tile columns (8 warps)

struct PadLayout {
    int PL, NP;
    size_t slice;                        // NP*NP
    __host__ __device__ size_t at(int i, int j, int ip, int jp, int ks) const
    {
        return (size_t)(i + PL) + (size_t)NP * (j + PL) + slice * (ip + (size_t)ks * jp);
    }
};

static PadLayout pad_layout(int ns, int ks)
{
    PadLayout L;
    L.PL = ks - 1;
    L.NP = ns + L.PL + XTY + L.PL;
    L.slice = (size_t)L.NP * L.NP;
    return L;
}

// 8-byte asynchronous global->shared copy; a false predicate writes zero.
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem, bool pred)
{
    unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    int sz = pred ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// Out[g,(i,ip)] = sum_(jp,j) Xd[g,(j,jp)] * rkb(i,j,ip,jp); epilogue UPDATE_HX 's'.
// A register-tiled FP64 GEMM: CTA tile 128 groups x 64 rows i of one ip, K = (j,jp)
// in steps of 16; 128 threads with 8x8 outputs each; operands double-buffered in
// shared memory by cp.async; the sum over K runs in the reference's order
// (jp outer, j inner) for every output.
constexpr int DG_TM = 128, DG_TN = 64, DG_TK = 16, DG_THREADS = 128;

__global__ void __launch_bounds__(DG_THREADS)
direct_gemm_kernel(int ns, int ks, int ng, const GroupDesc *__restrict__ gd, const double *__restrict__ Xd,
                   const double *__restrict__ rkbp, PadLayout L, double *hcc)
{
    __shared__ __align__(16) double As[2][DG_TK][DG_TM];
    __shared__ __align__(16) double Bs[2][DG_TK][DG_TN];
    const int i0 = blockIdx.x * DG_TN;
    const int ip = blockIdx.y;
    const int g0 = blockIdx.z * DG_TM;
    const int tx = threadIdx.x % 8, ty = threadIdx.x / 8;      // i: tx*8.., groups: ty*8..
    const size_t nn = (size_t)ns * ns, ldx = (size_t)ns * ks;
    // K steps: (jp, j0) with j0 < ns - jp
    int nsteps = 0;
    for (int jp = 0; jp < ks; jp++) nsteps += (ns - jp + DG_TK - 1) / DG_TK;
    auto load = [&](int buf, int step) {
        int jp = 0, s = step;
        for (;;) {
            int n = (ns - jp + DG_TK - 1) / DG_TK;
            if (s < n) break;
            s -= n;
            jp++;
        }
        int j0 = s * DG_TK, jmax = ns - jp;
        for (int q = threadIdx.x; q < DG_TK * DG_TM; q += DG_THREADS) {
            int kk = q % DG_TK, gg = q / DG_TK;
            int g = g0 + gg, j = j0 + kk;
            bool ok = g < ng && j < jmax;
            cp_async8(&As[buf][kk][gg], ok ? (const void *)(Xd + (size_t)g * ldx + j + (size_t)ns * jp) : (const void *)Xd, ok);
        }
        const double *R = rkbp + L.at(0, 0, ip, jp, ks);
        for (int q = threadIdx.x; q < DG_TK * DG_TN; q += DG_THREADS) {
            int ii = q % DG_TN, kk = q / DG_TN;
            int i = i0 + ii, j = j0 + kk;
            bool ok = i < ns && j < jmax;
            cp_async8(&Bs[buf][kk][ii], ok ? (const void *)(R + i + (size_t)L.NP * j) : (const void *)rkbp, ok);
        }
        cp_async_commit();
    };
    double acc[8][8];
#pragma unroll
    for (int r = 0; r < 8; r++)
#pragma unroll
        for (int c = 0; c < 8; c++) acc[r][c] = 0.0;
    load(0, 0);
    for (int st = 0; st < nsteps; st++) {
        int buf = st & 1;
        if (st + 1 < nsteps) { load(buf ^ 1, st + 1); cp_async_wait<1>(); }
        else cp_async_wait<0>();
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < DG_TK; kk++) {
            double a[8], b[8];
            const double2 *ap = reinterpret_cast<const double2 *>(&As[buf][kk][ty * 8]);
            const double2 *bp = reinterpret_cast<const double2 *>(&Bs[buf][kk][tx * 8]);
#pragma unroll
            for (int q = 0; q < 4; q++) {
                double2 va = ap[q], vb = bp[q];
                a[2 * q] = va.x; a[2 * q + 1] = va.y;
                b[2 * q] = vb.x; b[2 * q + 1] = vb.y;
            }
#pragma unroll
            for (int r = 0; r < 8; r++)
#pragma unroll
                for (int c = 0; c < 8; c++) acc[r][c] = fma(a[r], b[c], acc[r][c]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int r = 0; r < 8; r++) {
        int g = g0 + ty * 8 + r;
        if (g >= ng) continue;
        double *blk = hcc + (size_t)gd[g].blk * nn;
#pragma unroll
        for (int c = 0; c < 8; c++) {
            int i = i0 + tx * 8 + c;
            if (i + ip >= ns) continue;
            double v = acc[r][c];
            blk[i + (size_t)ns * (i + ip)] += v;
            if (ip > 0) blk[(i + ip) + (size_t)ns * i] += v;
        }
    }
}

// The direct contraction as one library GEMM: the multipole's table reshaped to
// the dense (ns ks) x (ns ks) matrix R3[(i,ip),(j,jp)] = rkb(i,j,ip,jp), then
// C[(i,ip), g] = sum_(j,jp) R3[(i,ip),(j,jp)] Xd[(j,jp), g] by cuBLAS DGEMM, then
// UPDATE_HX 's' of each group's band into its channel block.
__global__ void direct_table_kernel(int ns, int ks, const double *__restrict__ rkbp, PadLayout L,
                                    double *__restrict__ R3)
{
    const size_t nk = (size_t)ns * ks;
    const size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (q >= nk * nk) return;
    const int row = (int)(q % nk), colk = (int)(q / nk);
    const int i = row % ns, ip = row / ns, j = colk % ns, jp = colk / ns;
    R3[q] = rkbp[L.at(i, j, ip, jp, ks)];
}

// Thread (column c, offset o = row - c, |o| < ks): the band of column c is one
// contiguous run of 2ks-1 doubles, so a warp's read-modify-writes share sectors.
// Row c+o <= c holds the band element (i, i+ip) with i = c+o, ip = -o; row c+o > c
// its mirror (i+ip, i) with i = c, ip = o (UPDATE_HX 's', both triangles).
__global__ void direct_update_kernel(int ns, int ks, int ng, const GroupDesc *__restrict__ gd,
                                     const double *__restrict__ C, double *hcc)
{
    const int g = blockIdx.y;
    const int nb = 2 * ks - 1;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ng || q >= ns * nb) return;
    const int c = q / nb, o = q % nb - (ks - 1), r = c + o;
    if (r < 0 || r >= ns) return;
    const int i = o <= 0 ? r : c, ip = o <= 0 ? -o : o;
    const double v = C[i + (size_t)ns * ip + (size_t)ns * ks * g];
    double *blk = hcc + (size_t)gd[g].blk * ns * ns;
    blk[r + (size_t)ns * c] += v;
}

// ---------------------------------------------------------------------------
// The R^k table of the assembly pipeline, in a zero-margined layout:
//   rkbp[(i+PL) + NP*((j+PL) + NP*(ip + ks*jp))],  PL = ks-1 low margin,
//   NP = ns + PL + PH with PH = XTY + PL high margin (tile overhang),
// so the exchange kernel reads R for any shifted index of its tiles without
// bounds tests.  Values equal mrk_cell's (mrk_cell.f90:2): the cells of two
// disjoint interval ranges factorise, sum_iv sum_jv rkd1(iv) rkd2(jv) =
// M1(i,ip) M2(j,jp) with the band moments M1 = <B_i|r^k|B_i'>, M2 =
// <B_i|r^-(k+1)|B_i'>; pairs whose interval ranges overlap (|i-j| < ks) keep
// the diagonal cells and factorise the rest with running sums over iv.  All
// terms are positive, so the regrouping changes the result by a few ulp at most.
// ---------------------------------------------------------------------------
// M1(i,ip) = sum over cells of rkd1, M2 likewise (ascending interval order)
__global__ void band_moment_kernel(int ks, int ns, int nv, const double *__restrict__ rkd1,
                                   const double *__restrict__ rkd2, double *M1, double *M2)
{
    int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= ns * ks) return;
    int i = tid % ns, ip = tid / ns;
    const int ik = ks * (ks + 1) / 2;
    double a = 0.0, b = 0.0;
    if (i + ip < ns) {
        int lo = i + ip - (ks - 1); if (lo < 0) lo = 0;
        int hi = i < nv - 1 ? i : nv - 1;
        for (int iv = lo; iv <= hi; iv++) {
            int ih = i - iv, ii = ih * ks - ih * (ih - 1) / 2 + ip;
            a += rkd1[ii + (size_t)ik * iv];
            b += rkd2[ii + (size_t)ik * iv];
        }
    }
    M1[tid] = a;
    M2[tid] = b;
}

constexpr int PAD_TI = 32, PAD_TJ = 32, PAD_JT = PAD_TJ / 8;      // block tile, columns per thread

// Element (i, j) of one (ip, jp) slice whose interval ranges [iv_lo, iv_hi] and [jv_lo, jv_hi]
// overlap (only pairs with |i - j| < ks can): the diagonal cells rkd(ii,jj,jv) of the shared
// range, then sum_jv [ rkd2(jj,jv) sum_{iv<jv} rkd1(ii,iv) + rkd1(jj,jv) sum_{iv>jv} rkd2(ii,iv) ]
// with the iv sums running (ascending for iv < jv, descending for iv > jv).
template <int KS>
__device__ __forceinline__ double rkb_overlap(int i, int j, int ip, int jp, int iv_lo, int iv_hi, int jv_lo,
                                              int jv_hi, const double *__restrict__ rkd1,
                                              const double *__restrict__ rkd2, const double *__restrict__ rkd)
{
    constexpr int ks = KS, ik = KS * (KS + 1) / 2;
    auto cell = [&](int h, int p, int v) { return h * ks - h * (h - 1) / 2 + p + ik * v; };
    double v = 0.0;
    // the diagonal cells first: independent loads, unrolled so they overlap
    const int ov_lo = iv_lo > jv_lo ? iv_lo : jv_lo, ov_hi = iv_hi < jv_hi ? iv_hi : jv_hi;
#pragma unroll 4
    for (int jv = ov_lo; jv <= ov_hi; jv++) {
        const int ih = i - jv, jh = j - jv;
        v += __ldg(rkd + ih * ks - ih * (ih - 1) / 2 + ip +
                   (size_t)ik * (jh * ks - jh * (jh - 1) / 2 + jp + (size_t)ik * jv));
    }
    double lo_sum = 0.0;               // sum of rkd1(ii,iv) over iv < jv
    int ivn = iv_lo;
    for (int jv = jv_lo; jv <= jv_hi; jv++) {
        for (; ivn < jv && ivn <= iv_hi; ivn++) lo_sum += __ldg(rkd1 + cell(i - ivn, ip, ivn));
        v += lo_sum * __ldg(rkd2 + cell(j - jv, jp, jv));
    }
    double hi_sum = 0.0;               // sum of rkd2(ii,iv) over iv > jv
    ivn = iv_hi;
    for (int jv = jv_hi; jv >= jv_lo; jv--) {
        for (; ivn > jv && ivn >= iv_lo; ivn--) hi_sum += __ldg(rkd2 + cell(i - ivn, ip, ivn));
        v += hi_sum * __ldg(rkd1 + cell(j - jv, jp, jv));
    }
    return v;
}

// Everything of the table but the band |i - j| < ks of valid elements: the factorised products
// M1(i,ip) M2(j,jp) (or M1(j,jp) M2(i,ip)) and the zero margins.  rkb_band_kernel writes the band.
template <int KS>
__global__ void __launch_bounds__(256)
rkb_pad_kernel(int ns, int nv, PadLayout L, const double *__restrict__ M1, const double *__restrict__ M2,
               double *__restrict__ rkbp)
{
    constexpr int ks = KS;
    // the block's band moments (A: M1(i,ip), M2(i,ip) of its rows; B: M1(j,jp), M2(j,jp) of its columns)
    __shared__ double A1[PAD_TI], A2[PAD_TI], B1[PAD_TJ], B2[PAD_TJ];
    const int ipjp = blockIdx.z, ip = ipjp % ks, jp = ipjp / ks;
    const int i0 = (int)blockIdx.x * PAD_TI - L.PL, j0 = (int)blockIdx.y * PAD_TJ - L.PL;
    const int t = threadIdx.x + 32 * threadIdx.y;
    if (t < PAD_TI) {
        const int i = i0 + t;
        const bool ok = i >= 0 && i + ip < ns;
        A1[t] = ok ? M1[i + (size_t)ns * ip] : 0.0;
        A2[t] = ok ? M2[i + (size_t)ns * ip] : 0.0;
    } else if (t < PAD_TI + PAD_TJ) {
        const int j = j0 + t - PAD_TI;
        const bool ok = j >= 0 && j + jp < ns;
        B1[t - PAD_TI] = ok ? M1[j + (size_t)ns * jp] : 0.0;
        B2[t - PAD_TI] = ok ? M2[j + (size_t)ns * jp] : 0.0;
    }
    __syncthreads();
    const int r = threadIdx.x, pr = blockIdx.x * PAD_TI + r, i = pr - L.PL;
    if (pr >= L.NP) return;
    const bool irow = i >= 0 && i + ip < ns;
    const int iv_hi = i < nv - 1 ? i : nv - 1;
    double *out = rkbp + (size_t)pr + L.slice * ipjp;
#pragma unroll
    for (int u = 0; u < PAD_JT; u++) {
        const int c = threadIdx.y + 8 * u, pc = blockIdx.y * PAD_TJ + c, j = pc - L.PL;
        if (pc >= L.NP) break;
        double v = 0.0;
        if (irow && j >= 0 && j + jp < ns) {
            if (j - i < ks && i - j < ks) continue;        // the band: rkb_band_kernel
            int jv_lo = j + jp - (ks - 1); if (jv_lo < 0) jv_lo = 0;
            v = iv_hi < jv_lo ? A1[r] * B2[c] : B1[c] * A2[r];
        }
        out[(size_t)L.NP * pc] = v;
    }
}

// The band |i - j| < ks of one (ip, jp) slice: one warp per 32 consecutive i of one diagonal
// d = j - i, so the lanes of a warp share their loop structure (a tile of rkb_pad_kernel mixed
// band and factorised elements in one warp and waited on its slowest lane).  Same arithmetic, in
// the same order, as the product of the cells.
template <int KS>
__global__ void __launch_bounds__(256)
rkb_band_kernel(int ns, int nv, PadLayout L, const double *__restrict__ rkd1, const double *__restrict__ rkd2,
                const double *__restrict__ rkd, const double *__restrict__ M1, const double *__restrict__ M2,
                double *__restrict__ rkbp)
{
    constexpr int ks = KS;
    const int ipjp = blockIdx.z, ip = ipjp % ks, jp = ipjp / ks;
    const int d = (int)blockIdx.y - (ks - 1);
    const int i = ((int)blockIdx.x * 8 + (int)threadIdx.y) * 32 + (int)threadIdx.x, j = i + d;
    if (i >= ns || j < 0 || j >= ns || i + ip >= ns || j + jp >= ns) return;
    int iv_lo = i + ip - (ks - 1); if (iv_lo < 0) iv_lo = 0;
    const int iv_hi = i < nv - 1 ? i : nv - 1;
    int jv_lo = j + jp - (ks - 1); if (jv_lo < 0) jv_lo = 0;
    const int jv_hi = j < nv - 1 ? j : nv - 1;
    double v;
    if (iv_hi < jv_lo) v = M1[i + (size_t)ns * ip] * M2[j + (size_t)ns * jp];
    else if (jv_hi < iv_lo) v = M1[j + (size_t)ns * jp] * M2[i + (size_t)ns * ip];
    else v = rkb_overlap<KS>(i, j, ip, jp, iv_lo, iv_hi, jv_lo, jv_hi, rkd1, rkd2, rkd);
    rkbp[L.at(i, j, ip, jp, ks)] = v;
}

// ---------------------------------------------------------------------------
// exchange groups: a(x,y') = sum_(x',y) R(x,x',y,y') D_g(x',y), D_g = sum c p_a p_b^T
//
// One CTA per (XTX x XTY output tile, G groups), 8 warps.  Lane l owns row
// x = x0 + l (the contiguous rkb index, so R loads coalesce); warp w owns the
// XTYT columns y' = y0 + XTYT w + j.  For each row shift e the thread walks the
// column shift f with a sliding window of D values held in registers: per f
// step it loads XTYT R values (shared by its G groups, from L2, no bounds
// tests thanks to the zero margins) and one new D value per group from shared
// memory, and issues G*XTYT FMAs.  The group densities (with halo) are built
// once per CTA in shared memory from staged term vectors and never touch HBM.
// ---------------------------------------------------------------------------
constexpr int XTC = 16;                  // terms staged per chunk in the density build

template <int KS, int G>
__global__ void __launch_bounds__(256, 2)
exchange_kernel(int ns, int ng, PadLayout L, const GroupDesc *__restrict__ gd, const int *__restrict__ ca,
                const int *__restrict__ cb, const double *__restrict__ cv, const double *__restrict__ P,
                const double *__restrict__ rkbp, double *hcc)
{
    constexpr int HW = KS - 1, WX = XTX + 2 * HW, WY = XTY + 2 * HW;
    constexpr int NQ = (WX * WY + 255) / 256;          // density entries per thread
    extern __shared__ double sm[];
    double *Dsm = sm;                                   // [G][WY cols (y)][WX rows (x')]
    double *U = Dsm + (size_t)G * WX * WY;              // [XTC][WX]
    double *V = U + XTC * WX;                           // [XTC][WY]
    const int tiles_x = (ns + XTX - 1) / XTX;
    const int x0 = (blockIdx.x % tiles_x) * XTX, y0 = (blockIdx.x / tiles_x) * XTY;
    const int gbase = blockIdx.y * G;
    const int ngl = ng - gbase < G ? ng - gbase : G;
    // ---- group densities D(x', y) = sum_t (c_t p_a(x')) p_b(y) ----
    for (int gl = 0; gl < G; gl++) {
        double *D = Dsm + (size_t)gl * WX * WY;
        int ts = 0, te = 0;
        if (gl < ngl) { ts = gd[gbase + gl].start; te = gd[gbase + gl].end; }
        double acc[NQ];
#pragma unroll
        for (int q = 0; q < NQ; q++) acc[q] = 0.0;
        for (int t0 = ts; t0 < te; t0 += XTC) {
            int nt = te - t0 < XTC ? te - t0 : XTC;
            __syncthreads();
            for (int q = threadIdx.x; q < nt * WX; q += 256) {
                int t = q / WX, r = q % WX, xp = x0 - HW + r;
                U[t * WX + r] = (xp >= 0 && xp < ns) ? cv[t0 + t] * P[(size_t)ns * ca[t0 + t] + xp] : 0.0;
            }
            for (int q = threadIdx.x; q < nt * WY; q += 256) {
                int t = q / WY, c = q % WY, y = y0 - HW + c;
                V[t * WY + c] = (y >= 0 && y < ns) ? P[(size_t)ns * cb[t0 + t] + y] : 0.0;
            }
            __syncthreads();
#pragma unroll
            for (int q = 0; q < NQ; q++) {
                int e = threadIdx.x + 256 * q;
                if (e < WX * WY) {
                    int r = e % WX, c = e / WX;
                    double a = acc[q];
                    for (int t = 0; t < nt; t++) a = fma(U[t * WX + r], V[t * WY + c], a);
                    acc[q] = a;
                }
            }
        }
#pragma unroll
        for (int q = 0; q < NQ; q++) {
            int e = threadIdx.x + 256 * q;
            if (e < WX * WY) D[e] = acc[q];
        }
    }
    __syncthreads();
    // ---- main loop ----
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int x = x0 + lane, yb = y0 + XTYT * w;
    const size_t NPs = (size_t)L.NP;
    double acc[G][XTYT];
#pragma unroll
    for (int gl = 0; gl < G; gl++)
#pragma unroll
        for (int j = 0; j < XTYT; j++) acc[gl][j] = 0.0;
    // R(x,x',y,y') at rkbp[(min(x,x')+PL) + NP*(min(y,y')+PL) + slice*(|e| + KS|f|)]
    const double *Rbase = rkbp + L.PL + NPs * (yb + L.PL);
    for (int e = -HW; e <= HW; e++) {
        const int r1 = e >= 0 ? x : x + e;
        const int rr = lane + e + HW;
        const double *Re = Rbase + r1 + L.slice * (e >= 0 ? e : -e);
        double dwin[G][XTYT];
#pragma unroll
        for (int gl = 0; gl < G; gl++)
#pragma unroll
            for (int j = 0; j < XTYT; j++) dwin[gl][j] = Dsm[(size_t)gl * WX * WY + (XTYT * w + j) * WX + rr];
#pragma unroll
        for (int f = -HW; f <= HW; f++) {
            const double *Rp = Re + L.slice * KS * (f >= 0 ? f : -f) + (f < 0 ? (long)f * (long)NPs : 0);
            double R[XTYT];
#pragma unroll
            for (int j = 0; j < XTYT; j++) R[j] = __ldg(Rp + NPs * j);
#pragma unroll
            for (int gl = 0; gl < G; gl++)
#pragma unroll
                for (int j = 0; j < XTYT; j++) acc[gl][j] = fma(R[j], dwin[gl][j], acc[gl][j]);
            if (f < HW) {
#pragma unroll
                for (int gl = 0; gl < G; gl++) {
#pragma unroll
                    for (int j = 0; j < XTYT - 1; j++) dwin[gl][j] = dwin[gl][j + 1];
                    dwin[gl][XTYT - 1] = Dsm[(size_t)gl * WX * WY + (XTYT * w + XTYT + f + HW) * WX + rr];
                }
            }
        }
    }
    if (x >= ns) return;
    const size_t nn = (size_t)ns * ns;
    for (int gl = 0; gl < ngl; gl++) {
        double *blk = hcc + (size_t)gd[gbase + gl].blk * nn;
#pragma unroll
        for (int j = 0; j < XTYT; j++) {
            const int yp = yb + j;
            if (yp < ns) blk[x + (size_t)ns * yp] += acc[gl][j];
        }
    }
}

// ---------------------------------------------------------------------------
// Exchange groups through the rank structure of the group densities.
//
// D_g = sum_t c_t p_a p_b^T is a sum of outer products, so
//   a_g(x,y') = sum_(e,f) R(x,x+e,y'+f,y') D_g(x+e,y'+f)
//             = sum_t c_t Z[y'][x][a_t][b_t]
// with, for every orbital pair,
//   W[y'][x][e][b] = sum_f R(x,x+e,y'+f,y') p_b(y'+f)      (19 x norb per output)
//   Z[y'][x][a][b] = sum_e p_a(x+e) W[y'][x][e][b]         (norb x norb per output)
// The reference contracts every group separately (convol icase 3 on the group
// density, (2ks-1)^2 multiply-adds per output and group); here each output
// costs (2ks-1)^2 norb + (2ks-1) norb^2 multiply-adds once for all groups plus
// one multiply-add per coefficient -- about 8x fewer at the config-2 sizes.
// One CTA per (column y', XCH consecutive rows x): R for the CTA goes to shared
// memory once, W and Z stay in shared memory, and each group's XCH outputs of
// the row are written side by side.  Same sum as the gather kernel, grouped
// differently: results agree to rounding.
// ---------------------------------------------------------------------------
constexpr int XCH = 4;                  // rows x per CTA
constexpr int NORB_MAX = 32;            // orbitals the factored kernel handles
constexpr int ZLD = NORB_MAX + 1;       // padded leading dimension of Z rows
// stride of one row xi's Z block, odd so the XCH threads of a group (same term,
// different xi) read different shared-memory banks in the term loop
constexpr int ZXS = NORB_MAX * ZLD + 1;

// records (8-byte coefficient + 2-byte Z offset) that fit in the R and W tiles of a CTA
__host__ __device__ constexpr int xf_term_cap(int ks)
{
    return (int)(sizeof(double) * ((size_t)XCH * (2 * ks - 1) * (2 * ks - 1) + (size_t)XCH * (2 * ks - 1) * NORB_MAX) /
                 (sizeof(double) + sizeof(unsigned short)));
}

// The launch's groups in chunks whose records fit in the CTA's dead R/W area: a staged
// chunk's coefficients and Z offsets are copied to shared memory once per CTA (one
// coalesced pass) instead of every thread reading them through L1; a chunk holding one
// group larger than the area is read from global memory.
struct XChunk {
    int g0, g1;       // groups [g0, g1) of the launch
    int staged;
};

template <int KS>
__global__ void __launch_bounds__(256)
exchange_factored_kernel(int ns, int norb, int ng, PadLayout L, const GroupDesc *__restrict__ gd,
                         const XChunk *__restrict__ chunks, int nchunk, const unsigned short *__restrict__ zoff,
                         const double *__restrict__ cv, const double *__restrict__ P,
                         const double *__restrict__ rkbp, double *hcc)
{
    constexpr int HW = KS - 1, NE = 2 * KS - 1, PXR = XCH + 2 * HW;
    extern __shared__ double fsm[];
    double *Py = fsm;                                    // p_b(y'+f)          [f][b]
    double *Px = Py + NE * NORB_MAX;                     // p_a(x0-HW+r)       [r][a]
    double *Rs = Px + PXR * NORB_MAX;                    // R(x,x+e,y'+f,y')   [xi][e][f]
    double *Ws = Rs + XCH * NE * NE;                     // W                  [xi][e][b]
    double *Zs = Ws + XCH * NE * NORB_MAX;               // Z                  [xi][a][b]
    const int yp = blockIdx.y;
    const int x0 = blockIdx.x * XCH;
    const int tid = threadIdx.x;
    const size_t nn = (size_t)ns * ns;
    // the XCH outputs of a group's block lie in one 32-byte sector when ns is a multiple
    // of 4: pull them towards L2 now, so the update at the end finds them there
    if (x0 < ns)
        for (int g = tid; g < ng; g += 256)
            asm volatile("prefetch.global.L2 [%0];" ::"l"(hcc + (size_t)gd[g].blk * nn + x0 + (size_t)ns * yp));
    // ---- stage p(y'+f), p(x0-HW+r) and the CTA's R values ----
    for (int q = tid; q < NE * NORB_MAX; q += 256) {
        int f = q / NORB_MAX - HW, b = q % NORB_MAX, y = yp + f;
        Py[q] = (b < norb && y >= 0 && y < ns) ? P[y + (size_t)ns * b] : 0.0;
    }
    for (int q = tid; q < PXR * NORB_MAX; q += 256) {
        int r = q / NORB_MAX, a = q % NORB_MAX, xr = x0 - HW + r;
        Px[q] = (a < norb && xr >= 0 && xr < ns) ? P[xr + (size_t)ns * a] : 0.0;
    }
    for (int q = tid; q < XCH * NE * NE; q += 256) {
        int xi = q % XCH, ef = q / XCH, e = ef / NE - HW, f = ef % NE - HW;
        int x = x0 + xi;
        double v = 0.0;
        if (x < ns) {
            int r1 = e >= 0 ? x : x + e, r2 = f >= 0 ? yp : yp + f;
            v = rkbp[(size_t)(r1 + L.PL) + (size_t)L.NP * (r2 + L.PL) + L.slice * ((e >= 0 ? e : -e) + KS * (f >= 0 ? f : -f))];
        }
        Rs[(xi * NE + (e + HW)) * NE + (f + HW)] = v;
    }
    __syncthreads();
    // ---- W[xi][e][b] = sum_f R[xi][e][f] Py[f][b] ----
    for (int q = tid; q < XCH * NE * NORB_MAX; q += 256) {
        int b = q % NORB_MAX, xe = q / NORB_MAX;            // xe = xi*NE + e
        const double *r = Rs + xe * NE;
        double w = 0.0;
#pragma unroll
        for (int f = 0; f < NE; f++) w = fma(r[f], Py[f * NORB_MAX + b], w);
        Ws[q] = w;
    }
    __syncthreads();
    // ---- Z[xi][a][b] = sum_e Px[xi+e][a] W[xi][e][b], 2x4 register tiles ----
    for (int q = tid; q < XCH * (NORB_MAX / 2) * (NORB_MAX / 4); q += 256) {
        int xi = q / ((NORB_MAX / 2) * (NORB_MAX / 4)), rem = q % ((NORB_MAX / 2) * (NORB_MAX / 4));
        int a0 = (rem / (NORB_MAX / 4)) * 2, b0 = (rem % (NORB_MAX / 4)) * 4;
        double z[2][4] = {};
#pragma unroll
        for (int e = 0; e < NE; e++) {
            const double *pa = Px + (xi + e) * NORB_MAX + a0;
            const double *wb = Ws + (xi * NE + e) * NORB_MAX + b0;
            double av[2] = {pa[0], pa[1]};
            double bv[4] = {wb[0], wb[1], wb[2], wb[3]};
#pragma unroll
            for (int i = 0; i < 2; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) z[i][j] = fma(av[i], bv[j], z[i][j]);
        }
#pragma unroll
        for (int i = 0; i < 2; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) Zs[xi * ZXS + (a0 + i) * ZLD + b0 + j] = z[i][j];
    }
    __syncthreads();
    // ---- a_g(x, y') = sum_t c_t Z[xi][a_t][b_t]; UPDATE_HX 'x' ----
    // thread (g, xi): the XCH threads of a group read the same terms (broadcast); the
    // records of a staged chunk live in the R/W area, dead once Z is built
    double *tcv = Rs;
    unsigned short *tzo = (unsigned short *)(tcv + xf_term_cap(KS));
    for (int ci = 0; ci < nchunk; ci++) {
        const XChunk C = chunks[ci];
        const int tb = gd[C.g0].start;
        if (C.staged) {
            const int te = gd[C.g1 - 1].end;
            __syncthreads();                // the previous chunk's readers are done
            for (int t = tb + tid; t < te; t += 256) {
                tcv[t - tb] = cv[t];
                tzo[t - tb] = zoff[t];
            }
            __syncthreads();
        }
        for (int q = tid; q < (C.g1 - C.g0) * XCH; q += 256) {
            int g = C.g0 + q / XCH, xi = q % XCH, x = x0 + xi;
            if (x >= ns) continue;
            GroupDesc G = gd[g];
            double *dst = hcc + (size_t)G.blk * nn + x + (size_t)ns * yp;
            const double old = *dst;        // issued before the term loop so its latency overlaps it
            const double *Z = Zs + xi * ZXS;
            double acc = 0.0;
            if (C.staged) {
#pragma unroll 4
                for (int t = G.start - tb; t < G.end - tb; t++) acc = fma(tcv[t], Z[tzo[t]], acc);
            } else {
#pragma unroll 4
                for (int t = G.start; t < G.end; t++) acc = fma(cv[t], Z[zoff[t]], acc);
            }
            *dst = old + acc;
        }
    }
}

typedef void (*exchange_factored_fn)(int, int, int, PadLayout, const GroupDesc *, const XChunk *, int,
                                     const unsigned short *, const double *, const double *, const double *, double *);

// Z offset a*ZLD + b of every coefficient, so the term loop of the factored
// kernel reads 10 bytes per term (all CTAs of a launch re-read the terms)
__global__ void pack_terms_kernel(int ncoef, const int *__restrict__ ca, const int *__restrict__ cb,
                                  unsigned short *zoff)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < ncoef) zoff[t] = (unsigned short)(ca[t] * ZLD + cb[t]);
}

static size_t exchange_factored_smem(int ks)
{
    int NE = 2 * ks - 1, PXR = XCH + 2 * (ks - 1);
    return sizeof(double) * ((size_t)NE * NORB_MAX + (size_t)PXR * NORB_MAX + (size_t)XCH * NE * NE +
                             (size_t)XCH * NE * NORB_MAX + (size_t)XCH * ZXS);
}

static exchange_factored_fn exchange_factored_for(int ks)
{
    switch (ks) {
    case 2: return exchange_factored_kernel<2>;
    case 3: return exchange_factored_kernel<3>;
    case 4: return exchange_factored_kernel<4>;
    case 5: return exchange_factored_kernel<5>;
    case 6: return exchange_factored_kernel<6>;
    case 7: return exchange_factored_kernel<7>;
    case 8: return exchange_factored_kernel<8>;
    case 9: return exchange_factored_kernel<9>;
    case 10: return exchange_factored_kernel<10>;
    case 11: return exchange_factored_kernel<11>;
    case 12: return exchange_factored_kernel<12>;
    default: return nullptr;
    }
}

// ---------------------------------------------------------------------------
// Exchange groups of every multipole in one pass: the factored form above with
// its two contractions on the FP64 tensor pipe (m8n8k4 DMMA) and each channel
// block's strip written once.
//
// One CTA per (column y', XF consecutive rows x); warp w owns row x = x0 + w.
// For each multipole k that has exchange groups:
//   W[e][b] = sum_f R(x,x+e,y'+f,y') p_b(y'+f)     DMMA  M = e, N = b, K = f
//   Z[a][b] = sum_e p_a(x+e) W[e][b]               DMMA  M = a, N = b, K = e
//   acc[blk][w] += sum_t c_t Z[a_t][b_t]           one thread per (group, row)
// The R window of the next multipole is fetched by cp.async while Z and the
// terms of the current one run.  After the last multipole the XF x 1 strip of
// every channel block is written once (write mode: the kernel is the first to
// touch H, so no separate zeroing pass) or added to the caller's blocks.  A block
// has at most one exchange group per multipole, so the per-k updates of acc are
// race-free.  Operand tiles in shared memory use row strides of 4 mod 16 doubles,
// with which the fragment loads of each half-warp hit 16 distinct 8-byte banks.
// ---------------------------------------------------------------------------
constexpr int XF = 8;                   // rows per CTA (one warp each)

__host__ __device__ constexpr int stride4mod16(int n) { return n <= 4 ? 4 : ((n - 4 + 15) / 16) * 16 + 4; }

template <int KS> struct XFLayout {
    static constexpr int HW = KS - 1, NE = 2 * KS - 1;
    static constexpr int KT = (NE + 3) / 4;          // k-steps over f (W) and over e (Z)
    static constexpr int EP = 4 * KT;                // padded e / f range
    static constexpr int ME = (NE + 7) / 8;          // m-tiles over e (W)
    static constexpr int SR = stride4mod16(EP);      // row stride of R, p_b^T and W^T
    static constexpr int SP = stride4mod16(XF + EP - 1);   // row stride of p_a^T
    static constexpr int REG = ((32 * SR > NORB_MAX * ZLD ? 32 * SR : NORB_MAX * ZLD)) | 1;  // W^T, then Z, per row
    static constexpr int PY = 0;                     // p_b(y'+f-HW)      [b][f]
    static constexpr int PX = PY + NORB_MAX * SR;    // p_a(x0-HW+r)      [a][r]
    static constexpr int RS = PX + NORB_MAX * SP;    // R                 [w][e][f]
    static constexpr int RG = RS + XF * NE * SR;     // per-row region    [w][REG]
    static constexpr int ACC = RG + XF * REG;        // strip sums        [w][blk]
    static size_t smem_bytes(int nblk) { return sizeof(double) * ((size_t)ACC + (size_t)nblk * XF); }
};

struct XKRange {
    int k, g0, ng, pad;                  // multipole, first exchange group, group count
};

template <int KS>
__global__ void __launch_bounds__(32 * XF, 1)
exchange_fused_kernel(int ns, int norb, int nblk, int nact, const XKRange *__restrict__ kr, PadLayout L,
                      const double *__restrict__ rk0, size_t tstride, const GroupDesc *__restrict__ gd,
                      const unsigned short *__restrict__ zoff, const double *__restrict__ cv,
                      const double *__restrict__ P, double *hcc, int accumulate)
{
    using Y = XFLayout<KS>;
    constexpr int HW = Y::HW, NE = Y::NE, KT = Y::KT, EP = Y::EP, ME = Y::ME, SR = Y::SR, SP = Y::SP;
    extern __shared__ __align__(16) double xs[];
    double *PyT = xs + Y::PY, *PxT = xs + Y::PX, *Rs = xs + Y::RS, *acc = xs + Y::ACC;   // acc [row][blk]
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, lr = lane >> 2, lc = lane & 3;
    const int x0 = blockIdx.x * XF, yp = blockIdx.y;
    const int ntb = (norb + 7) / 8;
    double *reg = xs + Y::RG + w * Y::REG;
    // ---- orbital windows, zeroed R tile (padding columns stay zero) and strip sums ----
    for (int q = tid; q < NORB_MAX * SR; q += 32 * XF) {
        const int b = q / SR, f = q % SR, y = yp + f - HW;
        PyT[q] = (b < norb && f < NE && y >= 0 && y < ns) ? P[y + (size_t)ns * b] : 0.0;
    }
    for (int q = tid; q < NORB_MAX * SP; q += 32 * XF) {
        const int a = q / SP, r = q % SP, xr = x0 - HW + r;
        PxT[q] = (a < norb && xr >= 0 && xr < ns) ? P[xr + (size_t)ns * a] : 0.0;
    }
    for (int q = tid; q < XF * NE * SR; q += 32 * XF) Rs[q] = 0.0;
    for (int q = tid; q < nblk * XF; q += 32 * XF) acc[q] = 0.0;
    __syncthreads();
    // R(x,x+e',y'+f',y') of multipole kr[i].k for the CTA's rows, e' = e-HW, f' = f-HW
    auto fetch_r = [&](int i) {
        const double *T = rk0 + tstride * (size_t)kr[i].k;
        for (int q = tid; q < XF * NE * NE; q += 32 * XF) {
            const int wi = q % XF, ef = q / XF, e = ef / NE - HW, f = ef % NE - HW, x = x0 + wi;
            const int r1 = e >= 0 ? x : x + e, r2 = f >= 0 ? yp : yp + f;
            const bool ok = x < ns;
            const double *src = ok ? T + (size_t)(r1 + L.PL) + (size_t)L.NP * (r2 + L.PL) +
                                         L.slice * ((e >= 0 ? e : -e) + KS * (f >= 0 ? f : -f))
                                   : T;
            cp_async8(Rs + (wi * NE + (e + HW)) * SR + (f + HW), src, ok);
        }
        cp_async_commit();
    };
    if (nact > 0) fetch_r(0);
    for (int i = 0; i < nact; i++) {
        cp_async_wait<0>();
        __syncthreads();                 // R(i) in place; the previous multipole's terms are done
        // ---- W = R P_y on the tensor pipe; rows e >= NE of R are zero ----
        double aw[ME][4][2];
#pragma unroll
        for (int mt = 0; mt < ME; mt++)
#pragma unroll
            for (int nt = 0; nt < 4; nt++) aw[mt][nt][0] = aw[mt][nt][1] = 0.0;
        const double *Rw = Rs + w * NE * SR;
#pragma unroll
        for (int kk = 0; kk < KT; kk++) {
            double bf[4];
#pragma unroll
            for (int nt = 0; nt < 4; nt++) bf[nt] = PyT[(nt * 8 + lr) * SR + kk * 4 + lc];
#pragma unroll
            for (int mt = 0; mt < ME; mt++) {
                const int e = mt * 8 + lr;
                const double af = e < NE ? Rw[e * SR + kk * 4 + lc] : 0.0;
#pragma unroll
                for (int nt = 0; nt < 4; nt++)
                    if (nt < ntb) dmma::mma884(aw[mt][nt][0], aw[mt][nt][1], af, bf[nt]);
            }
        }
        __syncthreads();                 // every warp is done with R(i)
        if (i + 1 < nact) fetch_r(i + 1);
        // W^T [b][e] into this row's region (rows e < EP; e >= NE are zero)
#pragma unroll
        for (int mt = 0; mt < ME; mt++)
#pragma unroll
            for (int nt = 0; nt < 4; nt++)
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    const int e = mt * 8 + lr, b = nt * 8 + 2 * lc + j;
                    if (e < EP && nt < ntb) reg[b * SR + e] = aw[mt][nt][j];
                }
        __syncwarp();
        // ---- Z = P_x^T W ----
        double az[4][4][2];
#pragma unroll
        for (int mt = 0; mt < 4; mt++)
#pragma unroll
            for (int nt = 0; nt < 4; nt++) az[mt][nt][0] = az[mt][nt][1] = 0.0;
#pragma unroll
        for (int kk = 0; kk < KT; kk++) {
            double bf[4];
#pragma unroll
            for (int nt = 0; nt < 4; nt++) bf[nt] = nt < ntb ? reg[(nt * 8 + lr) * SR + kk * 4 + lc] : 0.0;
#pragma unroll
            for (int mt = 0; mt < 4; mt++) {
                if (mt >= ntb) continue;
                const double af = PxT[(mt * 8 + lr) * SP + w + kk * 4 + lc];
#pragma unroll
                for (int nt = 0; nt < 4; nt++)
                    if (nt < ntb) dmma::mma884(az[mt][nt][0], az[mt][nt][1], af, bf[nt]);
            }
        }
        __syncwarp();                    // W^T reads done before Z overwrites the region
#pragma unroll
        for (int mt = 0; mt < 4; mt++)
#pragma unroll
            for (int nt = 0; nt < 4; nt++)
#pragma unroll
                for (int j = 0; j < 2; j++)
                    if (mt < ntb && nt < ntb) reg[(mt * 8 + lr) * ZLD + nt * 8 + 2 * lc + j] = az[mt][nt][j];
        __syncthreads();                 // Z of every row in place
        // ---- acc[row][blk] += sum_t c_t Z_row[a_t][b_t]: a thread per group, all XF rows at once,
        //      so each coefficient record is read once per CTA ----
        const XKRange K = kr[i];
        const double *Z0 = xs + Y::RG;
        for (int gi = tid; gi < K.ng; gi += 32 * XF) {
            const GroupDesc G = gd[K.g0 + gi];
            double s[XF];
#pragma unroll
            for (int wi = 0; wi < XF; wi++) s[wi] = 0.0;
            int t = G.start;
            for (; t + 1 < G.end; t += 2) {
                const double c0 = __ldg(cv + t), c1 = __ldg(cv + t + 1);
                const int z0 = __ldg(zoff + t), z1 = __ldg(zoff + t + 1);
#pragma unroll
                for (int wi = 0; wi < XF; wi++)
                    s[wi] = fma(c1, Z0[wi * Y::REG + z1], fma(c0, Z0[wi * Y::REG + z0], s[wi]));
            }
            if (t < G.end) {
                const double c0 = __ldg(cv + t);
                const int z0 = __ldg(zoff + t);
#pragma unroll
                for (int wi = 0; wi < XF; wi++) s[wi] = fma(c0, Z0[wi * Y::REG + z0], s[wi]);
            }
#pragma unroll
            for (int wi = 0; wi < XF; wi++) acc[wi * nblk + G.blk] += s[wi];
        }
    }
    __syncthreads();
    // ---- each block's strip, once ----
    const size_t nn = (size_t)ns * ns;
    for (int q = tid; q < nblk * XF; q += 32 * XF) {
        const int blk = q / XF, wi = q % XF, x = x0 + wi;
        if (x >= ns) continue;
        double *dst = hcc + (size_t)blk * nn + x + (size_t)ns * yp;
        const double a = acc[wi * nblk + blk];
        *dst = accumulate ? *dst + a : a;
    }
}

typedef void (*exchange_fused_fn)(int, int, int, int, const XKRange *, PadLayout, const double *, size_t,
                                  const GroupDesc *, const unsigned short *, const double *, const double *,
                                  double *, int);

static exchange_fused_fn exchange_fused_for(int ks, size_t *smem_fixed)
{
#define XFCASE(K) case K: *smem_fixed = XFLayout<K>::smem_bytes(0); return exchange_fused_kernel<K>;
    switch (ks) {
    XFCASE(2) XFCASE(3) XFCASE(4) XFCASE(5) XFCASE(6) XFCASE(7) XFCASE(8) XFCASE(9) XFCASE(10) XFCASE(11) XFCASE(12)
    default: *smem_fixed = 0; return nullptr;
    }
#undef XFCASE
}

typedef void (*rkb_pad_fn)(int, int, PadLayout, const double *, const double *, double *);
typedef void (*rkb_band_fn)(int, int, PadLayout, const double *, const double *, const double *, const double *,
                            const double *, double *);

#define PADCASE(K) \
    case K: *band = rkb_band_kernel<K>; return rkb_pad_kernel<K>;
static rkb_pad_fn rkb_pad_for(int ks, rkb_band_fn *band)
{
    switch (ks) {
    PADCASE(2) PADCASE(3) PADCASE(4) PADCASE(5) PADCASE(6) PADCASE(7) PADCASE(8) PADCASE(9)
    PADCASE(10) PADCASE(11) PADCASE(12) PADCASE(13) PADCASE(14) PADCASE(15) PADCASE(16)
    default: *band = nullptr; return nullptr;
    }
}
#undef PADCASE

// band moments + zero-margined R^k table of multipole k (from its cell moments)
static int build_padded_table(const bsrg_basis *b, int k, const double *rkd1, const double *rkd2, const double *rkd,
                              double *M1, double *M2, double *rkbp, cudaStream_t s)
{
    const int ns = b->ns, ks = b->ks, nv = b->nv;
    const PadLayout PL = pad_layout(ns, ks);
    band_moment_kernel<<<(ns * ks + 127) / 128, 128, 0, s>>>(ks, ns, nv, rkd1, rkd2, M1, M2);
    dim3 gp((PL.NP + PAD_TI - 1) / PAD_TI, (PL.NP + PAD_TJ - 1) / PAD_TJ, ks * ks);
    rkb_band_fn band = nullptr;
    rkb_pad_fn fn = rkb_pad_for(ks, &band);
    if (!fn || !band) {
        set_error("R^k table: ks=%d outside the compiled range 2..%d", ks, BSRG_MAXKS);
        return BSRG_ERR_ARG;
    }
    fn<<<gp, dim3(32, 8), 0, s>>>(ns, nv, PL, M1, M2, rkbp);
    dim3 gb((unsigned)((ns + 255) / 256), (unsigned)(2 * ks - 1), (unsigned)(ks * ks));
    band<<<gb, dim3(32, 8), 0, s>>>(ns, nv, PL, rkd1, rkd2, rkd, M1, M2, rkbp);
    (void)k;
    return cuda_fail(cudaGetLastError(), "R^k table");
}

static int exchange_groups_per_cta(int ks) { return ks <= 12 ? 4 : 2; }

static size_t exchange_smem(int ks)
{
    int WX = XTX + 2 * (ks - 1), WY = XTY + 2 * (ks - 1);
    return sizeof(double) * ((size_t)exchange_groups_per_cta(ks) * WX * WY + (size_t)XTC * (WX + WY));
}

typedef void (*exchange_fn)(int, int, PadLayout, const GroupDesc *, const int *, const int *, const double *,
                            const double *, const double *, double *);

static exchange_fn exchange_kernel_for(int ks)
{
    switch (ks) {
    case 2: return exchange_kernel<2, 4>;
    case 3: return exchange_kernel<3, 4>;
    case 4: return exchange_kernel<4, 4>;
    case 5: return exchange_kernel<5, 4>;
    case 6: return exchange_kernel<6, 4>;
    case 7: return exchange_kernel<7, 4>;
    case 8: return exchange_kernel<8, 4>;
    case 9: return exchange_kernel<9, 4>;
    case 10: return exchange_kernel<10, 4>;
    case 11: return exchange_kernel<11, 4>;
    case 12: return exchange_kernel<12, 4>;
    case 13: return exchange_kernel<13, 2>;
    case 14: return exchange_kernel<14, 2>;
    case 15: return exchange_kernel<15, 2>;
    case 16: return exchange_kernel<16, 2>;
    default: return nullptr;
    }
}

// ---------------------------------------------------------------------------
// asymptotic coefficients (UPDATE_CF): acf(ich,jch,k) = sum_t c_t <p_a|r^k|p_b>
// one warp per direct group; bvmv (bvmv.f90:2, 's') as a warp reduction.
// ---------------------------------------------------------------------------
__global__ void acf_kernel(int ns, int ks, int nch, int k, int ng, const GroupDesc *__restrict__ gd,
                           const int *__restrict__ ca, const int *__restrict__ cb,
                           const double *__restrict__ cv, const double *__restrict__ P,
                           const double *__restrict__ rmk, double *acf)
{
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) / 32, lane = threadIdx.x % 32;
    if (warp >= ng) return;
    GroupDesc G = gd[warp];
    double CA = 0.0;
    for (int t = G.start; t < G.end; t++) {
        const double *x = P + (size_t)ns * ca[t], *y = P + (size_t)ns * cb[t];
        double s = 0.0;
        for (int q = lane; q < ns * ks; q += 32) {
            int i = q % ns, jp = q / ns;           // band (i, jp), element (i, i+jp-(ks-1))
            int j = i + jp - (ks - 1);
            if (j < 0) continue;
            double a = rmk[q];
            s += jp == ks - 1 ? a * x[i] * y[i] : a * (x[i] * y[j] + x[j] * y[i]);
        }
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        CA += cv[t] * s;
    }
    if (lane == 0) acf[(G.ich - 1) + (size_t)nch * ((G.jch - 1) + (size_t)nch * k)] += CA;
}

// ---------------------------------------------------------------------------
// workspace helpers
// ---------------------------------------------------------------------------
int ctx_reserve(bsrg_ctx *c, size_t bytes)
{
    if (c->ws_bytes >= bytes) return BSRG_OK;
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "workspace sync");
    if (c->ws) cudaFree(c->ws);
    c->ws = nullptr;
    c->ws_bytes = 0;
    size_t want = bytes + (bytes >> 3);
    e = cudaMalloc(&c->ws, want);
    if (e != cudaSuccess) return cuda_fail(e, "workspace alloc");
    c->ws_bytes = want;
    return BSRG_OK;
}

int ctx_reserve_pinned(bsrg_ctx *c, size_t bytes)
{
    if (c->pinned_bytes >= bytes) {
        cudaError_t e = cudaEventSynchronize(c->ev_stage);
        return cuda_fail(e, "pinned staging wait");
    }
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "pinned sync");
    if (c->pinned) cudaFreeHost(c->pinned);
    c->pinned = nullptr;
    c->pinned_bytes = 0;
    size_t want = bytes + (bytes >> 3);
    e = cudaMallocHost(&c->pinned, want);
    if (e != cudaSuccess) return cuda_fail(e, "pinned alloc");
    c->pinned_bytes = want;
    return BSRG_OK;
}

void stage_begin(bsrg_ctx *c, int stage)
{
    if (!c->timing) return;
    cudaEvent_t a, b;
    for (cudaEvent_t *ev : {&a, &b}) {
        if (!c->pool->empty()) { *ev = c->pool->back(); c->pool->pop_back(); }
        else cudaEventCreate(ev);
    }
    cudaEventRecord(a, c->stream);
    c->events->push_back({stage, a, b});
}

void stage_end(bsrg_ctx *c, int stage, int launches)
{
    if (!c->timing) return;
    for (auto it = c->events->rbegin(); it != c->events->rend(); ++it)
        if (it->stage == stage) {
            cudaEventRecord(it->stop, c->stream);
            break;
        }
    c->stage_launches[stage] += launches;
}

int stage_collect(bsrg_ctx *c)
{
    if (!c->timing || c->events->empty()) return BSRG_OK;
    for (auto &e : *c->events) {
        cudaError_t err = cudaEventSynchronize(e.stop);
        if (err != cudaSuccess) return cuda_fail(err, "stage timing");
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e.start, e.stop);
        c->stage_ms[e.stage] += ms;
        c->pool->push_back(e.start);
        c->pool->push_back(e.stop);
    }
    c->events->clear();
    return BSRG_OK;
}

}  // namespace bsrg

using namespace bsrg;

extern "C" {

int bsrg_ctx_set_timing(bsrg_ctx *c, int on)
{
    if (!c) { set_error("ctx_set_timing: null context"); return BSRG_ERR_ARG; }
    int rc = stage_collect(c);
    c->timing = on ? 1 : 0;
    return rc;
}

int bsrg_ctx_stage_times(bsrg_ctx *c, double *ms, int *launches, int n)
{
    if (!c || !ms) { set_error("ctx_stage_times: null argument"); return BSRG_ERR_ARG; }
    int rc = stage_collect(c);
    for (int q = 0; q < n && q < BSRG_NSTAGE; q++) {
        ms[q] = c->stage_ms[q];
        if (launches) launches[q] = c->stage_launches[q];
    }
    for (int q = 0; q < BSRG_NSTAGE; q++) { c->stage_ms[q] = 0.0; c->stage_launches[q] = 0; }
    return rc;
}

int bsrg_ctx_set_precision(bsrg_ctx *c, int mixed)
{
    if (!c) { set_error("ctx_set_precision: null context"); return BSRG_ERR_ARG; }
    if (mixed < 0 || mixed > 2) { set_error("ctx_set_precision: form %d is not 0, 1 or 2", mixed); return BSRG_ERR_ARG; }
    c->precision = mixed;
    return BSRG_OK;
}

int bsrg_ctx_stage_flops(bsrg_ctx *c, double *flops, int n)
{
    if (!c || !flops) { set_error("ctx_stage_flops: null argument"); return BSRG_ERR_ARG; }
    for (int q = 0; q < n && q < BSRG_NSTAGE; q++) flops[q] = c->stage_flops[q];
    for (int q = 0; q < BSRG_NSTAGE; q++) c->stage_flops[q] = 0.0;
    return BSRG_OK;
}

int bsrg_ctx_create(int device, void *stream, bsrg_ctx **out)
{
    if (!out) { set_error("ctx_create: null output"); return BSRG_ERR_ARG; }
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_fail(e, "ctx_create setDevice");
    bsrg_ctx *c = new bsrg_ctx();
    std::memset(c, 0, sizeof *c);
    c->device = device;
    c->stream = (cudaStream_t)stream;
    if (cublasCreate(&c->blas) != CUBLAS_STATUS_SUCCESS) {
        delete c;
        set_error("ctx_create: cublasCreate failed");
        return BSRG_ERR_SOLVER;
    }
    cublasSetStream(c->blas, c->stream);
    if (cusolverDnCreate(&c->solver) != CUSOLVER_STATUS_SUCCESS) {
        cublasDestroy(c->blas);
        delete c;
        set_error("ctx_create: cusolverDnCreate failed");
        return BSRG_ERR_SOLVER;
    }
    cusolverDnSetStream(c->solver, c->stream);
    cudaEventCreateWithFlags(&c->ev_stage, cudaEventDisableTiming);
    cudaEventRecord(c->ev_stage, c->stream);
    int prio_lo = 0, prio_hi = 0;
    cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
    if (cudaStreamCreateWithPriority(&c->aux_stream, cudaStreamNonBlocking, prio_hi) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->aux_ev[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->aux_ev[1], cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        c->aux_stream = nullptr;              // the band reduction then runs on one stream
    }
    c->events = new std::vector<bsrg_stage_event>();
    c->pool = new std::vector<cudaEvent_t>();
    c->last_ipsol = new std::vector<int>();
    c->pw_knots = new std::vector<double>();
    c->refine = 1;
    *out = c;
    return BSRG_OK;
}

int bsrg_ctx_destroy(bsrg_ctx *c)
{
    if (!c) return BSRG_OK;
    cudaStreamSynchronize(c->stream);
    if (c->ws) cudaFree(c->ws);
    if (c->pinned) cudaFreeHost(c->pinned);
    cudaEventDestroy(c->ev_stage);
    if (c->aux_stream) {
        cudaStreamSynchronize(c->aux_stream);
        cudaStreamDestroy(c->aux_stream);
        cudaEventDestroy(c->aux_ev[0]);
        cudaEventDestroy(c->aux_ev[1]);
    }
    for (auto &e : *c->events) { cudaEventDestroy(e.start); cudaEventDestroy(e.stop); }
    for (auto ev : *c->pool) cudaEventDestroy(ev);
    delete c->events;
    delete c->pool;
    delete c->last_ipsol;
    if (c->pw_buf) cudaFree(c->pw_buf);
    if (c->rf_buf) cudaFree(c->rf_buf);
    bsrg_basis_free(c->pw_basis);
    delete c->pw_knots;
    cusolverDnDestroy(c->solver);
    cublasDestroy(c->blas);
    delete c;
    return BSRG_OK;
}

size_t bsrg_ctx_workspace_bytes(const bsrg_ctx *c) { return c ? c->ws_bytes : 0; }

}  // extern "C"

// full = true: the whole SUB1 of the synthetic partial wave (zeroed blocks, the
// one-electron part, the groups, E_ch sb, symmetrisation); full = false: only
// I_data Case(6..9) accumulated into the caller's blocks and acf.
static int assemble_impl(bsrg_ctx *c, const bsrg_basis *b, double z, int nch, const int *lch, const double *ech,
                         int norb, const double *P, int kmax, int ncoef, const int *ck, const int *ctype,
                         const int *cich, const int *cjch, const int *ca, const int *cb, const double *cval,
                         double *hcc, double *scc, double *acf, bool full)
{
    if (!c || !b || (full && (!lch || !ech)) || !P || !hcc ||
        (ncoef > 0 && (!ck || !ctype || !cich || !cjch || !ca || !cb || !cval))) {
        set_error("assemble: null argument");
        return BSRG_ERR_ARG;
    }
    if (nch < 1 || norb < 1 || kmax < 0 || ncoef < 0) {
        set_error("assemble: bad sizes nch=%d norb=%d kmax=%d ncoef=%d", nch, norb, kmax, ncoef);
        return BSRG_ERR_ARG;
    }
    const int ns = b->ns, ks = b->ks, nv = b->nv, ik = ik_of(ks);
    cudaStream_t s = c->stream;
    // ---- group the coefficient records (the cmdata blocks of State_res) ----
    std::vector<std::vector<GroupDesc>> dgroups(kmax + 1), xgroups(kmax + 1);
    for (int t = 0; t < ncoef;) {
        int k = ck[t], ty = ctype[t], i = cich[t], j = cjch[t];
        if (k < 0 || k > kmax || (ty != 0 && ty != 1) || i < 1 || i > nch || j < 1 || j > i) {
            set_error("assemble: coefficient %d out of range (k=%d type=%d ich=%d jch=%d)", t, k, ty, i, j);
            return BSRG_ERR_ARG;
        }
        int t0 = t;
        while (t < ncoef && ck[t] == k && ctype[t] == ty && cich[t] == i && cjch[t] == j) {
            if (ca[t] < 0 || ca[t] >= norb || cb[t] < 0 || cb[t] >= norb) {
                set_error("assemble: orbital index out of range at coefficient %d", t);
                return BSRG_ERR_ARG;
            }
            t++;
        }
        if (t < ncoef) {
            long a0 = ((long)k * 2 + ty) * (long)(nch + 1) * (nch + 1) + (long)i * (nch + 1) + j;
            long a1 = ((long)ck[t] * 2 + ctype[t]) * (long)(nch + 1) * (nch + 1) + (long)cich[t] * (nch + 1) + cjch[t];
            if (a1 < a0) {
                set_error("assemble: coefficients not sorted by (k,type,ich,jch) at %d", t);
                return BSRG_ERR_ARG;
            }
        }
        GroupDesc g{t0, t, i * (i - 1) / 2 + j - 1, i, j};
        (ty == 0 ? dgroups : xgroups)[k].push_back(g);
    }
    size_t ngroups = 0, maxgd = 0;
    for (int k = 0; k <= kmax; k++) {
        ngroups += dgroups[k].size() + xgroups[k].size();
        maxgd = std::max(maxgd, dgroups[k].size());
    }
    // chunks of each multipole's exchange groups for the factored kernel's record staging
    std::vector<std::vector<XChunk>> xchunks(kmax + 1);
    size_t nchunks = 0;
    {
        const int cap = xf_term_cap(ks);
        for (int k = 0; k <= kmax; k++) {
            const std::vector<GroupDesc> &xg = xgroups[k];
            int g = 0, nx = (int)xg.size();
            while (g < nx) {
                int g1 = g;
                while (g1 < nx && xg[g1].end - xg[g].start <= cap) g1++;
                if (g1 == g) xchunks[k].push_back(XChunk{g, g + 1, 0});
                else xchunks[k].push_back(XChunk{g, g1, 1});
                g = xchunks[k].back().g1;
            }
            nchunks += xchunks[k].size();
        }
    }
    // exchange of every multipole in one pass (exchange_fused_kernel) when the orbitals and
    // the channel blocks' strip sums fit; BSRG_EXCHANGE_PER_K keeps one launch per multipole
    const size_t nblk = (size_t)nch * (nch + 1) / 2;
    size_t xfu_smem = 0;
    exchange_fused_fn xfu = nullptr;
    if (norb <= NORB_MAX && !getenv("BSRG_EXCHANGE_PER_K") && !getenv("BSRG_EXCHANGE_GATHER")) {
        xfu = exchange_fused_for(ks, &xfu_smem);
        xfu_smem += sizeof(double) * nblk * XF;
        int optin = 0;
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
        if (xfu && xfu_smem > (size_t)optin) xfu = nullptr;
    }
    std::vector<XKRange> kact;
    // ---- workspace ----
    size_t nn = (size_t)ns * ns;
    size_t need = 0;
    auto add = [&](size_t bytes) { need += ((bytes + 255) & ~(size_t)255) + 256; };
    add(sizeof(int) * (size_t)ncoef * 2);
    add(sizeof(double) * (size_t)ncoef);
    add(sizeof(GroupDesc) * ngroups);
    add(sizeof(XChunk) * std::max<size_t>(nchunks, 1));
    add(sizeof(int) * nch);
    add(sizeof(double) * nch);
    add(sizeof(double) * (size_t)ik * nv * 2);
    add(sizeof(double) * (size_t)ik * ik * nv);
    const PadLayout PL = pad_layout(ns, ks);
    const bsrg_tables *tabs = (c->tables && c->tables->basis == b && c->tables->kmax >= kmax) ? c->tables : nullptr;
    // the fused exchange reads every multipole's table in one launch
    const size_t ntab = xfu ? (size_t)kmax + 1 : 1;
    if (!tabs) add(sizeof(double) * PL.slice * ks * ks * ntab);
    add(sizeof(XKRange) * ((size_t)kmax + 1));
    add(sizeof(double) * maxgd * ns * ks);
    add(sizeof(double) * (size_t)ns * ks * 3);
    // direct contraction by the FP64 tensor-core GEMM (unless BSRG_DIRECT_SIMT selects the register-tiled kernel)
    const bool direct_blas = maxgd > 0 && !getenv("BSRG_DIRECT_SIMT");
    const size_t nk = (size_t)ns * ks;
    if (direct_blas) {
        add(sizeof(double) * nk * nk);
        add(sizeof(double) * nk * maxgd);
        add(sizeof(int) * 4);      // the tensor-core product's wait flag (mixed precision)
        if (c->precision == 1) add(ozaki_ws_bytes((int)nk, (int)maxgd, (int)nk, 8));   // its digit planes
    }
    add(sizeof(unsigned short) * (size_t)ncoef);
    int rc = ctx_reserve(c, need);
    if (rc != BSRG_OK) return rc;
    size_t host_bytes = sizeof(int) * (size_t)ncoef * 2 + sizeof(double) * (size_t)ncoef +
                        sizeof(GroupDesc) * ngroups + sizeof(XChunk) * nchunks + sizeof(int) * nch +
                        sizeof(double) * nch + sizeof(XKRange) * ((size_t)kmax + 1) + 64;
    rc = ctx_reserve_pinned(c, host_bytes);
    if (rc != BSRG_OK) return rc;
    Arena ar{(char *)c->ws, 0, c->ws_bytes};
    int *d_ca = ar.take<int>(ncoef), *d_cb = ar.take<int>(ncoef);
    double *d_cv = ar.take<double>(ncoef);
    GroupDesc *d_gd = ar.take<GroupDesc>(ngroups);
    XChunk *d_xc = ar.take<XChunk>(std::max<size_t>(nchunks, 1));
    int *d_lch = ar.take<int>(nch);
    double *d_ech = ar.take<double>(nch);
    double *rkd1 = ar.take<double>((size_t)ik * nv), *rkd2 = ar.take<double>((size_t)ik * nv);
    double *rkd = ar.take<double>((size_t)ik * ik * nv);
    double *rkbp = tabs ? nullptr : ar.take<double>(PL.slice * ks * ks * ntab);
    XKRange *d_kr = ar.take<XKRange>((size_t)kmax + 1);
    double *Xd = ar.take<double>(std::max<size_t>(maxgd, 1) * ns * ks);
    double *rmk = ar.take<double>((size_t)ns * ks);
    double *M1 = ar.take<double>((size_t)ns * ks), *M2 = ar.take<double>((size_t)ns * ks);
    unsigned short *d_zoff = ar.take<unsigned short>(std::max(ncoef, 1));
    double *R3 = direct_blas ? ar.take<double>(nk * nk) : nullptr;
    double *Cd = direct_blas ? ar.take<double>(nk * maxgd) : nullptr;
    int *d_tcerr = direct_blas ? ar.take<int>(4) : nullptr;
    const bool mixed = c->precision != 0;
    const size_t oz_bytes = direct_blas && c->precision == 1 ? ozaki_ws_bytes((int)nk, (int)maxgd, (int)nk, 8) : 0;
    char *oz_ws = oz_bytes ? ar.take<char>(oz_bytes) : nullptr;
    if (mixed && d_tcerr) {
        cudaError_t em = cudaMemsetAsync(d_tcerr, 0, sizeof(int) * 4, s);
        if (em != cudaSuccess) return cuda_fail(em, "assemble: mixed flag");
    }
    // stage host metadata through pinned memory, one copy
    char *hp = (char *)c->pinned;
    size_t o = 0;
    auto stage = [&](const void *src, size_t bytes) { std::memcpy(hp + o, src, bytes); size_t r = o; o += bytes; return r; };
    size_t o_ca = stage(ca, sizeof(int) * ncoef), o_cb = stage(cb, sizeof(int) * ncoef);
    size_t o_cv = stage(cval, sizeof(double) * ncoef);
    size_t o_gd = o;
    std::vector<size_t> doff(kmax + 1), xoff(kmax + 1);
    for (int k = 0; k <= kmax; k++) {
        doff[k] = (o - o_gd) / sizeof(GroupDesc);
        stage(dgroups[k].data(), sizeof(GroupDesc) * dgroups[k].size());
        xoff[k] = (o - o_gd) / sizeof(GroupDesc);
        stage(xgroups[k].data(), sizeof(GroupDesc) * xgroups[k].size());
    }
    size_t o_xc = o;
    std::vector<size_t> xcoff(kmax + 1);
    for (int k = 0; k <= kmax; k++) {
        xcoff[k] = (o - o_xc) / sizeof(XChunk);
        stage(xchunks[k].data(), sizeof(XChunk) * xchunks[k].size());
    }
    size_t o_lch = full ? stage(lch, sizeof(int) * nch) : 0, o_ech = full ? stage(ech, sizeof(double) * nch) : 0;
    for (int k = 0; k <= kmax; k++)
        if (!xgroups[k].empty()) kact.push_back(XKRange{k, (int)xoff[k], (int)xgroups[k].size(), 0});
    size_t o_kr = stage(kact.data(), sizeof(XKRange) * kact.size());
    cudaError_t e;
#define CP(dst, off, bytes) \
    if ((bytes) > 0 && (e = cudaMemcpyAsync(dst, hp + (off), bytes, cudaMemcpyHostToDevice, s)) != cudaSuccess) \
        return cuda_fail(e, "assemble upload");
    CP(d_ca, o_ca, sizeof(int) * ncoef);
    CP(d_cb, o_cb, sizeof(int) * ncoef);
    CP(d_cv, o_cv, sizeof(double) * ncoef);
    CP(d_gd, o_gd, sizeof(GroupDesc) * ngroups);
    CP(d_xc, o_xc, sizeof(XChunk) * nchunks);
    if (full) {
        CP(d_lch, o_lch, sizeof(int) * nch);
        CP(d_ech, o_ech, sizeof(double) * nch);
    }
    if (xfu) CP(d_kr, o_kr, sizeof(XKRange) * kact.size());
#undef CP
    cudaEventRecord(c->ev_stage, s);
    const size_t tstride = tabs ? tabs->table_doubles : PL.slice * ks * ks;
    const double *rk0 = tabs ? tabs->rkbp : rkbp;
    if (xfu) {
        // ---- the R^k tables of every multipole, then the exchange of all of them (first writer of H) ----
        if (!tabs)
            for (int k = 0; k <= kmax; k++) {
                if (dgroups[k].empty() && xgroups[k].empty()) continue;
                stage_begin(c, 0);
                rc = launch_rk_moments(b, k, rkd1, rkd2, rkd, s);
                if (rc != BSRG_OK) return rc;
                stage_end(c, 0, 3);
                stage_begin(c, 7);
                rc = build_padded_table(b, k, rkd1, rkd2, rkd, M1, M2, rkbp + tstride * k, s);
                if (rc != BSRG_OK) return rc;
                stage_end(c, 7, 2);
            }
        if ((e = smem_attr(xfu, (int)xfu_smem)) != cudaSuccess)
            return cuda_fail(e, "exchange (fused) smem");
    }
    if (xfu && (full || !kact.empty())) {
        stage_begin(c, 2);
        int launches = 1;
        if (!kact.empty()) {
            pack_terms_kernel<<<(ncoef + 255) / 256, 256, 0, s>>>(ncoef, d_ca, d_cb, d_zoff);
            launches++;
        }
        dim3 gx((ns + XF - 1) / XF, ns);
        xfu<<<gx, 32 * XF, xfu_smem, s>>>(ns, norb, (int)nblk, (int)kact.size(), d_kr, PL, rk0, tstride, d_gd,
                                          d_zoff, d_cv, P, hcc, full ? 0 : 1);
        stage_end(c, 2, launches);
        // executed arithmetic: the two contractions per output and multipole, one FMA per output and record
        const double NE = 2.0 * ks - 1.0;
        double nxt = 0.0;
        for (const XKRange &r : kact) nxt += (double)(xgroups[r.k].back().end - xgroups[r.k].front().start);
        c->stage_flops[2] += 2.0 * nn * ((double)kact.size() * (NE * NE * norb + NE * norb * norb) + nxt);
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "exchange (fused)");
    }
    // ---- one-electron part ----
    if (full) {
        if (!xfu && (e = cudaMemsetAsync(hcc, 0, sizeof(double) * nn * nblk, s)) != cudaSuccess)
            return cuda_fail(e, "memset hcc");
        if (scc && (e = cudaMemsetAsync(scc, 0, sizeof(double) * nn * nblk, s)) != cudaSuccess)
            return cuda_fail(e, "memset scc");
        if (acf && (e = cudaMemsetAsync(acf, 0, sizeof(double) * nch * nch * (kmax + 1), s)) != cudaSuccess)
            return cuda_fail(e, "memset acf");
        stage_begin(c, 3);
        dim3 g((ns * ks + 127) / 128, nch);
        one_electron_kernel<<<g, 128, 0, s>>>(ns, ks, nch, d_lch, z, b->db2, b->rm2, b->rm1, hcc);
        stage_end(c, 3);
    }
    // ---- two-electron groups, one multipole at a time ----
    const size_t xsm = exchange_smem(ks);
    const int xg = exchange_groups_per_cta(ks);
    exchange_fn xk = exchange_kernel_for(ks);
    if (!xk) { set_error("assemble: ks=%d unsupported", ks); return BSRG_ERR_ARG; }
    if ((e = smem_attr(xk, (int)xsm)) != cudaSuccess)
        return cuda_fail(e, "exchange smem");
    // the factored exchange handles up to NORB_MAX orbitals; BSRG_EXCHANGE_GATHER selects the gather kernel
    exchange_factored_fn xf = (norb <= NORB_MAX && !getenv("BSRG_EXCHANGE_GATHER")) ? exchange_factored_for(ks) : nullptr;
    const size_t xfsm = exchange_factored_smem(ks);
    if (xf && !xfu) {
        if ((e = smem_attr(xf, (int)xfsm)) != cudaSuccess)
            return cuda_fail(e, "exchange (factored) smem");
        if (ncoef > 0) {
            stage_begin(c, 2);
            pack_terms_kernel<<<(ncoef + 255) / 256, 256, 0, s>>>(ncoef, d_ca, d_cb, d_zoff);
            stage_end(c, 2, 1);
        }
    }
    for (int k = 0; k <= kmax; k++) {
        int nd = (int)dgroups[k].size(), nx = (int)xgroups[k].size();
        if (nd == 0 && nx == 0) continue;
        const double *rkbk = rkbp;
        if (tabs) {
            rkbk = tabs->rkbp + tabs->table_doubles * k;        // resident table of this multipole
        } else if (xfu) {
            rkbk = rkbp + PL.slice * ks * ks * k;               // built above with the exchange
        } else {
            stage_begin(c, 0);
            rc = launch_rk_moments(b, k, rkd1, rkd2, rkd, s);
            if (rc != BSRG_OK) return rc;
            stage_end(c, 0, 3);
            stage_begin(c, 7);
            rc = build_padded_table(b, k, rkd1, rkd2, rkd, M1, M2, rkbp, s);
            if (rc != BSRG_OK) return rc;
            stage_end(c, 7, 2);
        }
        if (nd > 0) {
            stage_begin(c, 1);
            const GroupDesc *gdd = d_gd + doff[k];
            dim3 g1((ns * ks + 127) / 128, nd);
            direct_density_kernel<<<g1, 128, 0, s>>>(ns, ks, nd, gdd, d_ca, d_cb, d_cv, P, Xd);
            if (direct_blas) {
                direct_table_kernel<<<(unsigned)((nk * nk + 255) / 256), 256, 0, s>>>(ns, ks, rkbk, PL, R3);
                // C = R Xd on the FP64 tensor pipe (dgemm.cu), or in the mixed-precision form from 8-bit
                // digits on tcgen05 (tc_ozaki.cu), or as the split-TF32 product (tc_mixed.cu)
                if (oz_ws)
                    rc = ozaki_gemm((int)nk, nd, (int)nk, 1.0, R3, (long)nk, Xd, (long)nk, 0.0, Cd, (long)nk, 8,
                                    oz_ws, oz_bytes, d_tcerr, s);
                else if (mixed)
                    rc = tf32x3_gemm((int)nk, nd, (int)nk, 1.0, R3, (long)nk, Xd, (long)nk, 0.0, Cd, (long)nk, d_tcerr,
                                     s);
                else
                    rc = dgemm(false, false, (int)nk, nd, (int)nk, 1.0, R3, (long)nk, Xd, (long)nk, 0.0, Cd,
                               (long)nk, s);
                if (rc != BSRG_OK) return rc;
                dim3 g4((unsigned)(((size_t)ns * (2 * ks - 1) + 127) / 128), nd);
                direct_update_kernel<<<g4, 128, 0, s>>>(ns, ks, nd, gdd, Cd, hcc);
            } else {
                dim3 g2((ns + DG_TN - 1) / DG_TN, ks, (nd + DG_TM - 1) / DG_TM);
                direct_gemm_kernel<<<g2, DG_THREADS, 0, s>>>(ns, ks, nd, gdd, Xd, rkbk, PL, hcc);
            }
            if (acf) {
                rc = launch_mrm(b, k, rmk, s);
                if (rc != BSRG_OK) return rc;
                acf_kernel<<<(nd * 32 + 127) / 128, 128, 0, s>>>(ns, ks, nch, k, nd, gdd, d_ca, d_cb, d_cv, P,
                                                                 rmk, acf);
            }
            stage_end(c, 1, (direct_blas ? 3 : 2) + (acf ? 2 : 0));
        }
        if (nx > 0 && !xfu) {
            stage_begin(c, 2);
            if (xf) {
                dim3 g3((ns + XCH - 1) / XCH, ns);
                xf<<<g3, 256, xfsm, s>>>(ns, norb, nx, PL, d_gd + xoff[k], d_xc + xcoff[k], (int)xchunks[k].size(),
                                         d_zoff, d_cv, P, rkbk, hcc);
            } else {
                int tiles = ((ns + XTX - 1) / XTX) * ((ns + XTY - 1) / XTY);
                dim3 g3(tiles, (nx + xg - 1) / xg);
                xk<<<g3, 256, xsm, s>>>(ns, nx, PL, d_gd + xoff[k], d_ca, d_cb, d_cv, P, rkbk, hcc);
            }
            stage_end(c, 2, 1);
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "assemble k-loop");
    }
    if (mixed && d_tcerr) {
        // the tensor-core product reports a device-side wait that ran out through this flag
        int hf = 0;
        cudaError_t em = cudaMemcpyAsync(&hf, d_tcerr, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (em == cudaSuccess) em = cudaStreamSynchronize(s);
        if (em != cudaSuccess) return cuda_fail(em, "assemble: mixed flag");
        if (hf == 2) { set_error("assemble: non-finite value in the direct contraction"); return BSRG_ERR_ARG; }
        if (hf) { set_error("assemble: a tensor-core wait timed out"); return BSRG_ERR_CUDA; }
    }
    // ---- target energies, overlap, symmetrisation ----
    if (!full) {
        rc = cuda_fail(cudaGetLastError(), "add_two_electron");
        if (rc == BSRG_OK) rc = stage_collect(c);
        return rc;
    }
    stage_begin(c, 3);
    {
        dim3 g((ns * ks + 127) / 128, nch);
        sb_update_kernel<<<g, 128, 0, s>>>(ns, ks, nch, d_ech, b->sb, hcc, scc);
        dim3 g2((ns * ns + 127) / 128, nch);
        symmetrize_diag_kernel<<<g2, 128, 0, s>>>(ns, nch, hcc);
    }
    stage_end(c, 3, 2);
    rc = cuda_fail(cudaGetLastError(), "assemble");
    if (rc == BSRG_OK) rc = stage_collect(c);
    return rc;
}

extern "C" {

int bsrg_assemble(bsrg_ctx *c, const bsrg_basis *b, double z, int nch, const int *lch, const double *ech,
                  int norb, const double *P, int kmax, int ncoef, const int *ck, const int *ctype,
                  const int *cich, const int *cjch, const int *ca, const int *cb, const double *cval,
                  double *hcc, double *scc, double *acf)
{
    return assemble_impl(c, b, z, nch, lch, ech, norb, P, kmax, ncoef, ck, ctype, cich, cjch, ca, cb, cval, hcc,
                         scc, acf, true);
}

int bsrg_add_two_electron(bsrg_ctx *c, const bsrg_basis *b, int nch, int norb, const double *P, int kmax,
                          int ncoef, const int *ck, const int *ctype, const int *cich, const int *cjch,
                          const int *ca, const int *cb, const double *cval, double *hcc, double *acf)
{
    return assemble_impl(c, b, 0.0, nch, nullptr, nullptr, norb, P, kmax, ncoef, ck, ctype, cich, cjch, ca, cb,
                         cval, hcc, nullptr, acf, false);
}

int bsrg_tables_create(bsrg_ctx *c, const bsrg_basis *b, int kmax, bsrg_tables **out)
{
    if (!c || !b || !out || kmax < 0 || kmax > 64) { set_error("tables_create: bad argument"); return BSRG_ERR_ARG; }
    const int ns = b->ns, ks = b->ks, nv = b->nv, ik = ik_of(ks);
    const PadLayout PL = pad_layout(ns, ks);
    bsrg_tables *t = new bsrg_tables();
    t->basis = b;
    t->kmax = kmax;
    t->table_doubles = PL.slice * ks * ks;
    cudaError_t e = cudaMalloc((void **)&t->rkbp, sizeof(double) * t->table_doubles * (kmax + 1));
    if (e != cudaSuccess) { delete t; return cuda_fail(e, "tables_create alloc"); }
    double *scratch = nullptr;
    size_t n1 = (size_t)ik * nv, n3 = (size_t)ik * ik * nv;
    e = cudaMalloc((void **)&scratch, sizeof(double) * (2 * n1 + n3 + 2 * (size_t)ns * ks));
    if (e != cudaSuccess) { cudaFree(t->rkbp); delete t; return cuda_fail(e, "tables_create scratch"); }
    int rc = BSRG_OK;
    for (int k = 0; k <= kmax && rc == BSRG_OK; k++) {
        rc = launch_rk_moments(b, k, scratch, scratch + n1, scratch + 2 * n1, c->stream);
        if (rc == BSRG_OK)
            rc = build_padded_table(b, k, scratch, scratch + n1, scratch + 2 * n1, scratch + 2 * n1 + n3,
                                    scratch + 2 * n1 + n3 + (size_t)ns * ks, t->rkbp + t->table_doubles * k, c->stream);
    }
    cudaError_t e2 = cudaStreamSynchronize(c->stream);
    cudaFree(scratch);
    if (rc == BSRG_OK && e2 != cudaSuccess) rc = cuda_fail(e2, "tables_create");
    if (rc != BSRG_OK) { cudaFree(t->rkbp); delete t; return rc; }
    *out = t;
    return BSRG_OK;
}

int bsrg_tables_free(bsrg_tables *t)
{
    if (!t) return BSRG_OK;
    cudaFree(t->rkbp);
    delete t;
    return BSRG_OK;
}

size_t bsrg_tables_bytes(const bsrg_tables *t) { return t ? sizeof(double) * t->table_doubles * (t->kmax + 1) : 0; }

int bsrg_ctx_use_tables(bsrg_ctx *c, const bsrg_tables *t)
{
    if (!c) { set_error("ctx_use_tables: null context"); return BSRG_ERR_ARG; }
    c->tables = t;
    return BSRG_OK;
}

}  // extern "C"
