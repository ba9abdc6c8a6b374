// bsrg_mrk_cell_noalloc: the R^k table without any device allocation.
//
// bsrg_mrk_cell allocates (and frees) scratch for the interval moments it
// expands into the table.  Some callers must not allocate device memory once
// they are running: a serving process that splits the whole HBM among its
// partial-wave solves at start-up has nothing left to hand out, and a
// cudaMalloc or cudaFree can stall every other stream of the device while it
// runs.  This entry point keeps the moments in a fixed array that lives inside
// the library instead.  It has no counterpart in the reference.
//
// The array is a file-scope static __device__ array, so every GPU that loads
// libbsrgpu.so holds it (BSRG_NOALLOC_SCRATCH_DOUBLES doubles, 6 MiB) until the
// process exits.  Host code cannot use the array's name as a device address;
// the first call on each device therefore looks the address up with
// cudaGetSymbolAddress while that device is current and caches it.  That
// first call should come before any stream capture on the device.
//
// All calls on a device share the one array and it keeps the last call's
// contents: two calls whose work overlaps on the GPU (different streams, or
// different host threads) race on it and must be serialised by the caller.
// Nothing in the array has to start at zero: every moment the expansion reads
// is written earlier in the same call.
//
// The call runs on the basis's device: if another device is current it is
// switched to b->device for the call and switched back afterwards.  The
// cached address belongs to the device's primary context; calls after a
// cudaDeviceReset of that device (which tears the context down) are not
// supported.
#include <mutex>

#include "bsrg_internal.h"

namespace bsrg {

static __device__ __align__(256) double g_noalloc_scratch[BSRG_NOALLOC_SCRATCH_DOUBLES];

static const int kMaxDevices = 64;
static double *g_scratch_ptr[kMaxDevices];
static std::mutex g_scratch_mu;

// device address of g_noalloc_scratch on device `dev`, which must be current
// (set up once per device)
static int scratch_address(int dev, double **out)
{
    cudaError_t e;
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("mrk_cell_noalloc: device %d beyond %d", dev, kMaxDevices);
        return BSRG_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "mrk_cell_noalloc: cudaGetSymbolAddress");
        g_scratch_ptr[dev] = (double *)p;
    }
    *out = g_scratch_ptr[dev];
    return BSRG_OK;
}

}  // namespace bsrg

using namespace bsrg;

extern "C" int bsrg_mrk_cell_noalloc(const bsrg_basis *b, int k, double *rkb, int ldp, void *stream)
{
    if (!b || !rkb) { set_error("mrk_cell_noalloc: null argument"); return BSRG_ERR_ARG; }
    if (ldp < b->ks) { set_error("mrk_cell_noalloc: ldp=%d < ks=%d", ldp, b->ks); return BSRG_ERR_ARG; }
    if (k < 0 || k > 64) { set_error("mrk_cell_noalloc: k=%d out of range", k); return BSRG_ERR_ARG; }
    const int ik = ik_of(b->ks);
    const size_t n1 = (size_t)ik * b->nv, n3 = (size_t)ik * ik * b->nv;
    const size_t need = 2 * n1 + n3;
    if (need > (size_t)BSRG_NOALLOC_SCRATCH_DOUBLES) {
        set_error("mrk_cell_noalloc: the moments need %zu doubles ((2*ik + ik^2)*nv with ik=%d, nv=%d) but the "
                  "built-in scratch holds %d; use bsrg_mrk_cell for this basis",
                  need, ik, b->nv, BSRG_NOALLOC_SCRATCH_DOUBLES);
        return BSRG_ERR_ARG;
    }
    int cur = 0;
    cudaError_t e = cudaGetDevice(&cur);
    if (e != cudaSuccess) return cuda_fail(e, "mrk_cell_noalloc: cudaGetDevice");
    if (cur != b->device && (e = cudaSetDevice(b->device)) != cudaSuccess)
        return cuda_fail(e, "mrk_cell_noalloc: cudaSetDevice");
    double *scratch = nullptr;
    int rc = scratch_address(b->device, &scratch);
    cudaStream_t s = (cudaStream_t)stream;
    if (rc == BSRG_OK) rc = launch_rk_moments(b, k, scratch, scratch + n1, scratch + 2 * n1, s);
    if (rc == BSRG_OK) rc = launch_mrk_cell(b, scratch, scratch + n1, scratch + 2 * n1, rkb, ldp, s);
    if (cur != b->device) cudaSetDevice(cur);
    return rc;
}
