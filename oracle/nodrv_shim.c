/* Host-memory stand-ins for the few CUDA runtime calls the reference CPU
 * backend makes through its pinned-memory allocator.  Used only to run
 * oracle/_ref/bin/parahpop_cpu in a container without a CUDA driver (test
 * infrastructure; never loaded on a machine with a GPU):
 *
 *   LD_PRELOAD=oracle/_ref/libnodrv_shim.so oracle/_ref/bin/parahpop_cpu ...
 */
#include <stdlib.h>
#include <string.h>

typedef int cudaError_t;
typedef void* cudaStream_t;

cudaError_t cudaMallocHost(void** p, size_t n) {
    *p = aligned_alloc(256, (n + 255) / 256 * 256 + 256);
    return *p ? 0 : 2;
}
cudaError_t cudaHostAlloc(void** p, size_t n, unsigned int flags) {
    (void)flags;
    return cudaMallocHost(p, n);
}
cudaError_t cudaFreeHost(void* p) { free(p); return 0; }
cudaError_t cudaHostRegister(void* p, size_t n, unsigned int f) { (void)p; (void)n; (void)f; return 0; }
cudaError_t cudaHostUnregister(void* p) { (void)p; return 0; }
cudaError_t cudaMemcpy(void* d, const void* s, size_t n, int kind) { (void)kind; memmove(d, s, n); return 0; }
cudaError_t cudaMemcpyAsync(void* d, const void* s, size_t n, int kind, cudaStream_t st) {
    (void)kind; (void)st; memmove(d, s, n); return 0;
}
cudaError_t cudaGetLastError(void) { return 0; }
cudaError_t cudaPeekAtLastError(void) { return 0; }
