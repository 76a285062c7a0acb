// egg_selfcheck.cu -- the reference-arithmetic sieve tiles' division, checked against the device's
// correctly rounded division on caller-chosen operands.
//
// A Hessenberg step of the reference-arithmetic tiles divides every row's entry by the same pivot.
// The tiles take one correctly rounded reciprocal of the pivot per step and finish each quotient
// with Markstein's corrections (div_rn_shared, egg_sieve_tile.cuh); the reference's `/`
// (src/hafnian.jl:235-238) is the correctly rounded quotient.  This entry point evaluates both on
// the device for n operand pairs, so a test can compare them bit for bit on operands the sieve's
// own workloads seldom reach (huge and tiny magnitudes, subnormals, signed zeros, infinities, NaN).
#include "egg_internal.cuh"
#include "egg_sieve_tile.cuh"

namespace egg {

static constexpr int64_t kSelfCheckMax = (int64_t)1 << 26;

static __global__ void division_check_kernel(const double *__restrict__ a, const double *__restrict__ b, int64_t n,
                                             double *__restrict__ q_shared, double *__restrict__ q_rn)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double x = b[i];
        // As a step of the tiles forms it: the reciprocal only when the pivot is in range.
        const bool x_ok = div_scale_ok(x);
        const double y = x_ok ? __drcp_rn(x) : 0.0;
        q_shared[i] = div_rn_shared(a[i], x, y, x_ok);
        q_rn[i] = __ddiv_rn(a[i], x);
    }
}

}  // namespace egg

using namespace egg;

extern "C" int egg_selfcheck_division(const double *a, const double *b, int64_t n, double *q_shared, double *q_rn)
{
    if (n < 0 || n > kSelfCheckMax)
        return fail(EGG_ERR_ARGUMENT, "egg_selfcheck_division: n must be in [0, 2^26], got " + std::to_string(n));
    if (n == 0) return EGG_OK;
    if (!a || !b || !q_shared || !q_rn) return fail(EGG_ERR_ARGUMENT, "egg_selfcheck_division: null pointer");
    const size_t bytes = (size_t)n * sizeof(double);
    double *d = nullptr;
    EGG_CUDA_TRY(cudaMalloc(&d, 4 * bytes));
    double *da = d, *db = d + n, *dq = d + 2 * n, *dr = d + 3 * n;
    int rc = EGG_OK;
    cudaError_t e = cudaMemcpy(da, a, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(db, b, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        const int threads = 256;
        const int64_t want = (n + threads - 1) / threads;
        const unsigned blocks = (unsigned)(want < 4096 ? want : 4096);
        division_check_kernel<<<blocks, threads>>>(da, db, n, dq, dr);
        count_launch();
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(q_shared, dq, bytes, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(q_rn, dr, bytes, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) rc = fail(EGG_ERR_CUDA, std::string("egg_selfcheck_division: ") + cudaGetErrorString(e));
    cudaFree(d);
    return rc;
}
