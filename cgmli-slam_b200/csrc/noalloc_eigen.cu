// Allocation-free variant of the dense eigensolver behind cgmli_marg_eigen.
//
// Who needs it: a process that shares the GPU with latency-critical work (the
// tracking front end of a SLAM pipeline, or a serving loop) often cannot let
// the backend call cudaMalloc / cudaFree - cudaFree synchronizes the whole
// device and stalls every other stream - and a process whose device memory is
// owned by another allocator (a caching allocator holding the budget) may not
// be able to obtain new memory at all.  cgmli_marg_eigen copies host arrays
// through a grow-only device workspace it allocates; this entry point takes
// device arrays from the caller and keeps the solver's work arrays in one
// fixed, file-scope device array instead, so it allocates nothing.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/cgmli_backend.h"

namespace cgmli {
void launchDenseEigen(const double* H, int n, double* work, double* evals, double* evecs, int* status, cudaStream_t s);
int setLastError(int code, const char* message);  // message for cgmli_last_error(); returns code
}  // namespace cgmli

namespace {
// Largest matrix order the fixed scratch holds.
constexpr int kNoAllocMaxN = CGMLI_MARG_EIGEN_NOALLOC_MAX_N;
// Scratch layout (doubles): Jacobi matrix n*n | eigenvectors n*n | eigenvalues
// 2n (sorted, then the unsorted copy) | status word.  Sized for n = kNoAllocMaxN
// (about 1 MiB); every GPU that loads the library holds it until the process exits.
constexpr size_t kScratchDoubles = 2ull * kNoAllocMaxN * kNoAllocMaxN + 2ull * kNoAllocMaxN + 8;
static __device__ __align__(256) double g_eigenScratch[kScratchDoubles];

// Device address of g_eigenScratch per device.  In host code the symbol name
// only stands in for the device array; its address must be asked from the runtime.
constexpr int kMaxDevices = 64;
double* g_scratchPtr[kMaxDevices] = {};
std::mutex g_scratchMutex;
}  // namespace

using cgmli::launchDenseEigen;
using cgmli::setLastError;

extern "C" {

int cgmli_marg_eigen_noalloc(const double* H, int n, double* eigenvalues, double* eigenvectors, void* stream) {
    if (!H || !eigenvalues || !eigenvectors || n < 1) {
        return setLastError(CGMLI_E_INVALID, "eigen (no-alloc): null device pointers or n < 1");
    }
    if (n > kNoAllocMaxN) {
        return setLastError(CGMLI_E_LIMIT, "eigen (no-alloc): n above CGMLI_MARG_EIGEN_NOALLOC_MAX_N (256); use cgmli_marg_eigen");
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        return setLastError(CGMLI_E_CUDA, "eigen (no-alloc): no current CUDA device");
    }
    double* scratch = nullptr;
    {
        // once per device, with that device current: look up the array's device address
        std::lock_guard<std::mutex> lock(g_scratchMutex);
        if (!g_scratchPtr[dev]) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_eigenScratch) != cudaSuccess || !p) {
                (void)cudaGetLastError();
                return setLastError(CGMLI_E_CUDA, "eigen (no-alloc): cudaGetSymbolAddress of the scratch array failed");
            }
            g_scratchPtr[dev] = static_cast<double*>(p);
        }
        scratch = g_scratchPtr[dev];
    }
    const size_t nn = (size_t)n * n;
    double* work = scratch;               // 2 n^2: Jacobi matrix and eigenvectors
    double* evals = scratch + 2 * nn;     // 2 n
    int* status = reinterpret_cast<int*>(evals + 2 * n);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // the status word keeps the previous call's value: clear it; the rest is fully rewritten
    if (cudaMemsetAsync(status, 0, sizeof(int), s) != cudaSuccess) {
        return setLastError(CGMLI_E_CUDA, "eigen (no-alloc): cudaMemsetAsync failed");
    }
    launchDenseEigen(H, n, work, evals, eigenvectors, status, s);
    int st = 0;
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(eigenvalues, evals, n * sizeof(double), cudaMemcpyDeviceToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(&st, status, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) {
        return setLastError(CGMLI_E_CUDA, "eigen (no-alloc): CUDA launch or copy failed");
    }
    if (st != CGMLI_OK) return setLastError(st, "eigen (no-alloc): non-finite eigenvalue");
    return CGMLI_OK;
}

}  // extern "C"
