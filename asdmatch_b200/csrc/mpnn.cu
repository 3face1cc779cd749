// Learned cardinality estimator: a 3-layer message-passing network over
// (sub-)query graphs, BF16 weights and activations with FP32 accumulation,
// forward, backward and Adam on the device.  The GEMMs run on the tcgen05
// tensor cores (tc_gemm.cuh).
#include <cstring>
#include <memory>
#include <vector>

#include "device.cuh"
#include "tc_gemm.cuh"

using namespace asdm;

// Test entry for the tensor-core GEMM: C[M][N] = sum_k A[m][k] * B[n][k]
// (bf16 bit patterns in, fp32 out; host arrays).
extern "C" int asdm_gemm_bf16(int M, int N, int K, const uint16_t *A, const uint16_t *B, float *C) {
    clear_error();
    if (M <= 0 || N <= 0 || K <= 0 || !A || !B || !C) return fail(ASDM_ERR_INVALID, "bad GEMM arguments");
    int dev = 0, sms = 0;
    ASDM_TRY(device_setup(&dev, &sms));
    cudaStream_t s;
    ASDM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    __nv_bfloat16 *dA = nullptr, *dB = nullptr;
    float *dC = nullptr;
    unsigned int *dErr = nullptr;
    int rc = ASDM_OK;
    do {
        if ((rc = dalloc(&dA, (uint64_t)M * K, s)) || (rc = dalloc(&dB, (uint64_t)N * K, s)) ||
            (rc = dalloc(&dC, (uint64_t)M * N, s)) || (rc = dalloc(&dErr, 1, s)))
            break;
        if (cudaMemcpyAsync(dA, A, (size_t)M * K * 2, cudaMemcpyHostToDevice, s) ||
            cudaMemcpyAsync(dB, B, (size_t)N * K * 2, cudaMemcpyHostToDevice, s) ||
            cudaMemsetAsync(dErr, 0, 4, s)) {
            rc = fail(ASDM_ERR_CUDA, "GEMM upload failed");
            break;
        }
        if (cudaFuncSetAttribute(tc::gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kSmemBytes)) {
            rc = fail(ASDM_ERR_CUDA, "GEMM shared-memory opt-in failed");
            break;
        }
        tc::Operand a{dA, K, 1, M}, b{dB, K, 1, N};
        dim3 grid((M + tc::kTileM - 1) / tc::kTileM, (N + tc::kTileN - 1) / tc::kTileN);
        tc::gemm_kernel<<<grid, tc::kThreads, tc::kSmemBytes, s>>>(a, b, M, N, K, dC, N, nullptr, 0, dErr);
        ::asdm::count_launch();
        unsigned int err = 0;
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpyAsync(C, dC, (size_t)M * N * 4, cudaMemcpyDeviceToHost, s) ||
            cudaMemcpyAsync(&err, dErr, 4, cudaMemcpyDeviceToHost, s) || cudaStreamSynchronize(s)) {
            rc = fail(ASDM_ERR_CUDA, "GEMM failed: %s", cudaGetErrorString(cudaGetLastError()));
            break;
        }
        if (err) rc = fail(ASDM_ERR_INTERNAL, "tensor-core wait ran out");
    } while (false);
    dfree(dA, s);
    dfree(dB, s);
    dfree(dC, s);
    dfree(dErr, s);
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    return rc;
}
