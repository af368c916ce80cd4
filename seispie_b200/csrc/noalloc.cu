// fwi_misfit_noalloc: the misfit / adjoint-source entry point without any
// caller-provided scratch.
//
// fwi_misfit needs a device buffer for its per-block FP64 partial sums, which
// the caller allocates.  Some callers cannot allocate device memory while they
// run: an application that hands all device memory to its own pool at start-up
// and forbids cudaMalloc afterwards, or a time-critical loop in which
// cudaMalloc / cudaFree would synchronise the device and stall work queued on
// other streams.  For them this entry point keeps the partial sums in a fixed
// array inside the library (FWI_MISFIT_NOALLOC_MAX_PARTIALS doubles, 1 MiB,
// held on every device that loads the library until the process exits).
//
// Set-up: every call looks up the array's device address on the current
// device with cudaGetSymbolAddress (cheap, allocates nothing), so the address
// is never stale, also after cudaDeviceReset.  The first call on a device may
// load the library's device code there; make it before any stream capture.
// The array is shared by every call:
// calls whose work overlaps on the GPU (other streams, other host threads)
// race on it, so issue them in order on one stream.  It keeps the last call's
// partial sums; nothing needs clearing, because every call writes each partial
// sum before its final reduction reads it.
#include "common.cuh"

namespace fwi {

int launch_misfit(const float *data, const float *syn, float *adstf, double *misfit, double *partial, int nshots,
                  int nrec, int nt, double dt, cudaStream_t st, bool grad);
long long misfit_partials(int nrec, int nt);

static __device__ __align__(256) double g_misfit_scratch[FWI_MISFIT_NOALLOC_MAX_PARTIALS];

// Device address of g_misfit_scratch on the current device, looked up on
// every call.  In host code the array's name only stands in for the symbol;
// a kernel given it directly would read host memory or fault.
static int misfit_scratch(double **out) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_misfit_scratch);
    if (e != cudaSuccess)
        return set_error(FWI_ECUDA, "fwi_misfit_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    *out = static_cast<double *>(p);
    return 0;
}

}  // namespace fwi

extern "C" int fwi_misfit_noalloc(const float *data, const float *syn, float *adstf, double *misfit, int nshots,
                                  int nrec, int nt, double dt, void *stream) {
    using namespace fwi;
    if (!(data && syn && adstf && misfit)) return set_error(FWI_EINVAL, "fwi_misfit_noalloc: NULL pointer");
    if (!(nshots >= 1 && nshots <= 65535 && nrec >= 0 && nrec <= 65535 && nt >= 0))
        return set_error(FWI_EINVAL, "fwi_misfit_noalloc: nshots in [1, 65535], nrec in [0, 65535], nt >= 0");
    const long long need = (long long)nshots * misfit_partials(nrec, nt);
    if (need > FWI_MISFIT_NOALLOC_MAX_PARTIALS)
        return set_error(FWI_ERANGE,
                         "fwi_misfit_noalloc: %d shots x %d receivers x %d samples need %lld partial sums; the fixed "
                         "scratch holds %d (nshots * nrec * ceil(nt/256) must not exceed it); use fwi_misfit",
                         nshots, nrec, nt, need, (int)FWI_MISFIT_NOALLOC_MAX_PARTIALS);
    if (nrec == 0 || nt == 0) {
        cudaError_t e = cudaMemsetAsync(misfit, 0, sizeof(double) * nshots, (cudaStream_t)stream);
        return e == cudaSuccess ? 0 : set_error(FWI_ECUDA, "fwi_misfit_noalloc: %s", cudaGetErrorString(e));
    }
    double *scratch = nullptr;
    int rc = misfit_scratch(&scratch);
    if (rc) return rc;
    return launch_misfit(data, syn, adstf, misfit, scratch, nshots, nrec, nt, dt, (cudaStream_t)stream, false);
}
