// egg_noalloc.cu -- a sieve entry point that allocates no device memory.
//
// Some callers cannot let a library call cudaMalloc.  A process whose device memory is owned by
// another allocator (a framework that reserves most of the GPU up front, or a caching allocator
// that must account for every byte) can see a stray cudaMalloc fail or fragment its pool.  A
// latency-critical loop that has finished its set-up may not allocate at all.  For them this file
// keeps the sieve's scratch -- its small instance tables and the per-warp double-double partial
// sums -- in one fixed array compiled into the library, and the caller supplies the input matrix and
// the output slot in device memory.
//
// Limits and behaviour:
//   * The scratch array holds kNoAllocScratchBytes (4 MiB).  It lives on every GPU that loads the
//     library, for the life of the process.  A sieve whose tables and partials need more is refused
//     with EGG_ERR_TOO_LARGE and a message giving both sizes (edge counts up to 32 fit).
//   * The first call on a device looks up, with that device current, the device addresses of this
//     array and of the library's binomial table (cudaGetSymbolAddress; both are module globals with
//     their contents in the image, so nothing is uploaded and no stream is touched) and caches them
//     per device; make that first call before capturing any stream.
//   * Every call uses the same array, and each call overwrites what it reads: the tables are copied
//     in and every partial-sum slot is written by its warp before the final reduction reads it, so
//     nothing has to start at zero.  Calls whose device work overlaps (on different streams, or from
//     different host threads) race on the array and must not be issued.
#include "egg_perdevice.h"
#include "egg_sieve.cuh"

namespace egg {

static constexpr size_t kNoAllocScratchBytes = (size_t)4 << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

struct NoAllocSlot {
    void *addr;   // device address of g_noalloc_scratch on that device
    int num_sms;
};
static PerDevice<NoAllocSlot> g_noalloc;

// Address of the scratch array on the current device (set up on the first call there).
static int noalloc_scratch(void **ptr, int *num_sms)
{
    int dev = -1;
    EGG_CUDA_TRY(cudaGetDevice(&dev));
    NoAllocSlot slot{nullptr, 0};
    int rc = g_noalloc.get(dev, &slot, [](int d, NoAllocSlot *out) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(EGG_ERR_CUDA, std::string("cudaGetSymbolAddress(fixed scratch): ") + cudaGetErrorString(e));
        int sms = 0;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d);
        if (e != cudaSuccess || sms <= 0)
            return fail(EGG_ERR_CUDA, std::string("cudaDeviceGetAttribute(SM count): ") + cudaGetErrorString(e));
        *out = NoAllocSlot{p, sms};
        return (int)EGG_OK;
    });
    if (rc == PerDevice<NoAllocSlot>::kBadDevice)
        return fail(EGG_ERR_NO_DEVICE, "device index " + std::to_string(dev) + " out of range for the fixed scratch");
    if (rc) return rc;
    *ptr = slot.addr;
    *num_sms = slot.num_sms;
    return EGG_OK;
}

}  // namespace egg

using namespace egg;

extern "C" int egg_sieve_device_noalloc(int dtype, int prec, const void *Ax, int64_t E, const int64_t *edge_reps,
                                        int glynn, void *out, void *stream)
{
    if (dtype != EGG_F64 && dtype != EGG_C128) return fail(EGG_ERR_ARGUMENT, "the sieve runs in Float64 or ComplexF64");
    if (E < 0 || E > 32) return fail(EGG_ERR_TOO_LARGE, "the device sieve supports up to 32 edges (N <= 64)");
    if (!out || (E > 0 && (!Ax || !edge_reps))) return fail(EGG_ERR_ARGUMENT, "null argument");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return fail(EGG_ERR_NO_DEVICE, "no CUDA device");
    }
    FixedScratch fs;
    int rc = noalloc_scratch(&fs.ptr, &fs.num_sms);
    if (rc) return rc;
    fs.bytes = kNoAllocScratchBytes;
    int32_t g = glynn ? 1 : 0;
    int64_t e = E;
    int64_t zero = 0;
    return sieve_batch_run(dtype, prec, 1, E, Ax, &e, E > 0 ? edge_reps : &zero, &g, out, (cudaStream_t)stream, &fs);
}
