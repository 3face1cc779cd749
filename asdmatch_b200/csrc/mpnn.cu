// Learned cardinality estimator: a 3-layer message-passing network over
// (sub-)query graphs, BF16 weights and activations with FP32 accumulation,
// forward, backward and Adam on the device.  The GEMMs run on the tcgen05
// tensor cores (tc_gemm.cuh).
#include <algorithm>
#include <cmath>
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

// ---------------------------------------------------------------------------
// The estimator.  For a graph (a sub-query) with node features x (F <= 128,
// zero-padded to 128):
//   H0 = x;  for l = 0, 1, 2:  X_l = [H_l | sum_{w in N(v)} H_l(w)]   (N x 256, bf16)
//                               Z_l = X_l W_l^T + b_l                  (tensor cores, fp32)
//                               H_{l+1} = relu(Z_l)
//   y = (sum_v H_3(v)) . w_o + b_o        (predicted log(1 + cardinality))
// trained with mean squared error and Adam, all on the device; the three
// matrix products per layer of the forward and backward passes (X W^T,
// dZ^T X, dZ W) go through gemm_kernel.
namespace asdm {
namespace est {

constexpr int kH = 128, kIn = 2 * kH, kLayers = 3;
constexpr int kT = 256;

__global__ void build_x(const float *__restrict__ H, const uint32_t *__restrict__ adj_off,
                        const uint32_t *__restrict__ adj, int n, __nv_bfloat16 *__restrict__ X) {
    // one thread per (node, feature)
    const long long total = (long long)n * kH;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const int v = (int)(i / kH), f = (int)(i % kH);
        float s = 0.f;
        for (uint32_t e = adj_off[v]; e < adj_off[v + 1]; ++e) s += H[(long long)adj[e] * kH + f];
        X[(long long)v * kIn + f] = __float2bfloat16(H[i]);
        X[(long long)v * kIn + kH + f] = __float2bfloat16(s);
    }
}

__global__ void relu_copy(const float *__restrict__ Z, float *__restrict__ H, long long total) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x)
        H[i] = fmaxf(Z[i], 0.f);
}

// g[graph] = sum of H3 over the graph's nodes, in node order (deterministic);
// one thread per (graph, feature)
__global__ void readout_sum(const float *__restrict__ H, const uint32_t *__restrict__ goff,
                            const uint32_t *__restrict__ gnodes, int ng, float *__restrict__ g) {
    const long long total = (long long)ng * kH;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const long long G = i / kH;
        const int f = (int)(i % kH);
        float s = 0.f;
        for (uint32_t j = goff[G]; j < goff[G + 1]; ++j) s += H[(long long)gnodes[j] * kH + f];
        g[i] = s;
    }
}

// y[G] = g[G] . w_o + b_o ; warp per graph
__global__ void readout_out(const float *__restrict__ g, const float *__restrict__ wo, const float *__restrict__ bo,
                            int ng, float *__restrict__ y) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= ng) return;
    float s = 0.f;
    for (int f = lane; f < kH; f += 32) s += g[(long long)warp * kH + f] * wo[f];
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) y[warp] = s + bo[0];
}

// dy = 2 (y - t) / ng; loss += (y - t)^2 / ng; grads of w_o, b_o; dg = dy * w_o
__global__ void loss_grad(const float *__restrict__ y, const float *__restrict__ t, const float *__restrict__ g,
                          const float *__restrict__ wo, int ng, float *__restrict__ dy, float *__restrict__ loss,
                          float *__restrict__ dwo, float *__restrict__ dbo) {
    for (int G = blockIdx.x * blockDim.x + threadIdx.x; G < ng; G += gridDim.x * blockDim.x) {
        const float r = y[G] - t[G];
        dy[G] = 2.f * r / ng;
        atomicAdd(loss, r * r / ng);
        atomicAdd(dbo, dy[G]);
        for (int f = 0; f < kH; ++f) atomicAdd(&dwo[f], dy[G] * g[(long long)G * kH + f]);
    }
}

// dH3[v] = dy[graph(v)] * w_o
__global__ void readout_back(const float *__restrict__ dy, const float *__restrict__ wo, const uint32_t *__restrict__ gid,
                             int n, float *__restrict__ dH) {
    const long long total = (long long)n * kH;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x)
        dH[i] = dy[gid[i / kH]] * wo[i % kH];
}

// dZ = dH * (Z > 0) as bf16; db += dZ (column sums)
__global__ void relu_back(const float *__restrict__ dH, const float *__restrict__ Z, int n, __nv_bfloat16 *__restrict__ dZ,
                          float *__restrict__ db) {
    __shared__ float part[kH];
    for (int f = threadIdx.x; f < kH; f += blockDim.x) part[f] = 0.f;
    __syncthreads();
    const long long total = (long long)n * kH;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const float d = Z[i] > 0.f ? dH[i] : 0.f;
        dZ[i] = __float2bfloat16(d);
        atomicAdd(&part[i % kH], d);
    }
    __syncthreads();
    for (int f = threadIdx.x; f < kH; f += blockDim.x) atomicAdd(&db[f], part[f]);
}

// dH_l[v] = dX[v][:H] + sum_{w in N(v)} dX[w][H:]
__global__ void x_back(const float *__restrict__ dX, const uint32_t *__restrict__ adj_off, const uint32_t *__restrict__ adj,
                       int n, float *__restrict__ dH) {
    const long long total = (long long)n * kH;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const int v = (int)(i / kH), f = (int)(i % kH);
        float s = dX[(long long)v * kIn + f];
        for (uint32_t e = adj_off[v]; e < adj_off[v + 1]; ++e) s += dX[(long long)adj[e] * kIn + kH + f];
        dH[i] = s;
    }
}

__global__ void adam(float *__restrict__ p, const float *__restrict__ gr, float *__restrict__ m, float *__restrict__ v,
                     long long n, float lr, float b1t, float b2t, __nv_bfloat16 *__restrict__ pb) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float g = gr[i];
        m[i] = 0.9f * m[i] + 0.1f * g;
        v[i] = 0.999f * v[i] + 0.001f * g * g;
        const float mh = m[i] / (1.f - b1t), vh = v[i] / (1.f - b2t);
        p[i] -= lr * mh / (sqrtf(vh) + 1e-8f);
        if (pb) pb[i] = __float2bfloat16(p[i]);
    }
}

// x_in[v][f] = x[v][f] for f < F, 0 above (the first layer's width is 128)
__global__ void pad_x(const float *__restrict__ x, uint32_t F, int n, float *__restrict__ x_in) {
    const long long total = (long long)n * kH;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const uint32_t f = (uint32_t)(i % kH);
        x_in[i] = f < F ? x[(i / kH) * F + f] : 0.f;
    }
}

__global__ void to_bf16(const float *__restrict__ a, __nv_bfloat16 *__restrict__ b, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = __float2bfloat16(a[i]);
}

unsigned grid_of(long long n) { return (unsigned)std::max<long long>(1, std::min<long long>((n + kT - 1) / kT, 148LL * 16)); }

}  // namespace est
}  // namespace asdm

// parameter block layout (fp32): W_0..W_2 (128 x 256 each), b_0..b_2 (128), w_o (128), b_o (1)
struct asdm_estimator {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint32_t in_features = 0;
    long long nparam = 0;
    float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;   // params, grads, Adam moments
    __nv_bfloat16 *wb = nullptr;                                     // bf16 copies of W_0..W_2
    unsigned int *err = nullptr;
    long long step = 0;
    // batch workspace (grown on demand)
    int cap_nodes = 0, cap_graphs = 0;
    uint64_t cap_edges = 0;
    float *x_stage = nullptr, *x_in = nullptr, *H = nullptr, *Z = nullptr, *dH = nullptr, *dX = nullptr, *gsum = nullptr, *y = nullptr,
          *t = nullptr, *dy = nullptr, *loss = nullptr;
    __nv_bfloat16 *X = nullptr, *dZ = nullptr;
    uint32_t *adj_off = nullptr, *adj = nullptr, *gid = nullptr;
    uint32_t *goff = nullptr, *gnodes = nullptr;  // nodes of each graph, ascending

    static constexpr long long kW = (long long)asdm::est::kH * asdm::est::kIn;
    float *W(int l) { return p + l * kW; }
    float *bias(int l) { return p + 3 * kW + l * asdm::est::kH; }
    float *wo() { return p + 3 * kW + 3 * asdm::est::kH; }
    float *bo() { return wo() + asdm::est::kH; }
    float *gW(int l) { return g + l * kW; }
    float *gbias(int l) { return g + 3 * kW + l * asdm::est::kH; }
    float *gwo() { return g + 3 * kW + 3 * asdm::est::kH; }
    float *gbo() { return gwo() + asdm::est::kH; }
};

namespace {

using namespace asdm;
using namespace asdm::est;

void free_batch(asdm_estimator *e) {
    cudaStream_t s = e->stream;
    dfree(e->x_stage, s); dfree(e->x_in, s); dfree(e->H, s); dfree(e->Z, s); dfree(e->dH, s); dfree(e->dX, s); dfree(e->gsum, s);
    dfree(e->y, s); dfree(e->t, s); dfree(e->dy, s); dfree(e->loss, s); dfree(e->X, s); dfree(e->dZ, s);
    dfree(e->adj_off, s); dfree(e->adj, s); dfree(e->gid, s); dfree(e->goff, s); dfree(e->gnodes, s);
    e->cap_nodes = e->cap_graphs = 0;
    e->cap_edges = 0;
}

int ensure_batch(asdm_estimator *e, int nodes, int graphs, uint64_t edges) {
    if (nodes <= e->cap_nodes && graphs <= e->cap_graphs && edges <= e->cap_edges) return ASDM_OK;
    free_batch(e);
    cudaStream_t s = e->stream;
    const int N = std::max(nodes, 1), G = std::max(graphs, 1);
    const uint64_t E = std::max<uint64_t>(edges, 1);
    ASDM_TRY(dalloc(&e->x_stage, (uint64_t)N * e->in_features, s));
    ASDM_TRY(dalloc(&e->x_in, (uint64_t)N * kH, s));
    ASDM_TRY(dalloc(&e->H, (uint64_t)(kLayers + 1) * N * kH, s));
    ASDM_TRY(dalloc(&e->Z, (uint64_t)kLayers * N * kH, s));
    ASDM_TRY(dalloc(&e->dH, (uint64_t)N * kH, s));
    ASDM_TRY(dalloc(&e->dX, (uint64_t)N * kIn, s));
    ASDM_TRY(dalloc(&e->gsum, (uint64_t)G * kH, s));
    ASDM_TRY(dalloc(&e->y, G, s));
    ASDM_TRY(dalloc(&e->t, G, s));
    ASDM_TRY(dalloc(&e->dy, G, s));
    ASDM_TRY(dalloc(&e->loss, 1, s));
    ASDM_TRY(dalloc(&e->X, (uint64_t)kLayers * N * kIn, s));
    ASDM_TRY(dalloc(&e->dZ, (uint64_t)N * kH, s));
    ASDM_TRY(dalloc(&e->adj_off, (uint64_t)N + 1, s));
    ASDM_TRY(dalloc(&e->adj, E, s));
    ASDM_TRY(dalloc(&e->gid, N, s));
    ASDM_TRY(dalloc(&e->goff, (uint64_t)G + 1, s));
    ASDM_TRY(dalloc(&e->gnodes, N, s));
    e->cap_nodes = N;
    e->cap_graphs = G;
    e->cap_edges = E;
    return ASDM_OK;
}

int gemm(asdm_estimator *e, tc::Operand A, tc::Operand B, int M, int N, int K, float *C, long long ldc,
         const float *bias) {
    dim3 grid((M + tc::kTileM - 1) / tc::kTileM, (N + tc::kTileN - 1) / tc::kTileN);
    tc::gemm_kernel<<<grid, tc::kThreads, tc::kSmemBytes, e->stream>>>(A, B, M, N, K, C, ldc, bias, 0, e->err);
    ::asdm::count_launch();
    ASDM_CUDA(cudaGetLastError());
    return ASDM_OK;
}

// Forward pass for a batch already uploaded; leaves y on the device.
int forward(asdm_estimator *e, int n, int ng) {
    cudaStream_t s = e->stream;
    const long long nh = (long long)n * kH;
    ASDM_CUDA(cudaMemcpyAsync(e->H, e->x_in, nh * sizeof(float), cudaMemcpyDeviceToDevice, s));
    for (int l = 0; l < kLayers; ++l) {
        float *Hl = e->H + l * nh, *Hn = e->H + (l + 1) * nh, *Zl = e->Z + l * nh;
        __nv_bfloat16 *Xl = e->X + (long long)l * n * kIn;
        build_x<<<grid_of(nh), kT, 0, s>>>(Hl, e->adj_off, e->adj, n, Xl);
        ::asdm::count_launch();
        tc::Operand a{Xl, kIn, 1, n};
        tc::Operand b{e->wb + l * asdm_estimator::kW, kIn, 1, kH};
        ASDM_TRY(gemm(e, a, b, n, kH, kIn, Zl, kH, e->bias(l)));
        relu_copy<<<grid_of(nh), kT, 0, s>>>(Zl, Hn, nh);
        ::asdm::count_launch();
    }
    readout_sum<<<grid_of((long long)ng * kH), kT, 0, s>>>(e->H + kLayers * nh, e->goff, e->gnodes, ng, e->gsum);
    readout_out<<<(ng * 32 + kT - 1) / kT, kT, 0, s>>>(e->gsum, e->wo(), e->bo(), ng, e->y);
    ::asdm::count_launch();
    ::asdm::count_launch();
    ASDM_CUDA(cudaGetLastError());
    return ASDM_OK;
}

int upload_batch(asdm_estimator *e, int n, int ng, const float *x, const uint32_t *adj_off, const uint32_t *adj,
                 const uint32_t *node_graph) {
    const uint64_t ne = adj_off[n];
    ASDM_TRY(ensure_batch(e, n, ng, ne));
    cudaStream_t s = e->stream;
    for (int v = 0; v < n; ++v)
        if (node_graph[v] >= (uint32_t)ng) return fail(ASDM_ERR_INVALID, "node %d belongs to graph %u >= %d", v, node_graph[v], ng);
    for (uint64_t i = 0; i < ne; ++i)
        if (adj[i] >= (uint32_t)n) return fail(ASDM_ERR_INVALID, "adjacency entry out of range");
    // nodes grouped by graph (counting sort, stable)
    std::vector<uint32_t> goff((size_t)ng + 1, 0), gnodes((size_t)n);
    for (int v = 0; v < n; ++v) ++goff[node_graph[v] + 1];
    for (int G = 0; G < ng; ++G) goff[G + 1] += goff[G];
    {
        std::vector<uint32_t> at(goff.begin(), goff.end() - 1);
        for (int v = 0; v < n; ++v) gnodes[at[node_graph[v]]++] = (uint32_t)v;
    }
    ASDM_CUDA(cudaMemcpyAsync(e->x_stage, x, (size_t)n * e->in_features * 4, cudaMemcpyHostToDevice, s));
    pad_x<<<grid_of((long long)n * kH), kT, 0, s>>>(e->x_stage, e->in_features, n, e->x_in);
    ::asdm::count_launch();
    ASDM_CUDA(cudaMemcpyAsync(e->adj_off, adj_off, (size_t)(n + 1) * 4, cudaMemcpyHostToDevice, s));
    if (ne) ASDM_CUDA(cudaMemcpyAsync(e->adj, adj, ne * 4, cudaMemcpyHostToDevice, s));
    ASDM_CUDA(cudaMemcpyAsync(e->gid, node_graph, (size_t)n * 4, cudaMemcpyHostToDevice, s));
    ASDM_CUDA(cudaMemcpyAsync(e->goff, goff.data(), goff.size() * 4, cudaMemcpyHostToDevice, s));
    ASDM_CUDA(cudaMemcpyAsync(e->gnodes, gnodes.data(), gnodes.size() * 4, cudaMemcpyHostToDevice, s));
    ASDM_CUDA(cudaStreamSynchronize(s));  // host staging vectors go out of scope
    return ASDM_OK;
}

int check_err(asdm_estimator *e) {
    unsigned int err = 0;
    ASDM_CUDA(cudaMemcpyAsync(&err, e->err, 4, cudaMemcpyDeviceToHost, e->stream));
    ASDM_CUDA(cudaStreamSynchronize(e->stream));
    if (err) return fail(ASDM_ERR_INTERNAL, "tensor-core wait ran out");
    return ASDM_OK;
}

}  // namespace

extern "C" int asdm_est_create(uint32_t in_features, uint64_t seed, asdm_estimator **out) {
    clear_error();
    if (!out || in_features == 0 || in_features > (uint32_t)kH) return fail(ASDM_ERR_INVALID, "1..128 input features");
    auto e = std::make_unique<asdm_estimator>();
    int sms = 0;
    ASDM_TRY(device_setup(&e->device, &sms));
    ASDM_CUDA(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
    ASDM_CUDA(cudaFuncSetAttribute(tc::gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kSmemBytes));
    e->in_features = in_features;
    e->nparam = 3 * asdm_estimator::kW + 3 * kH + kH + 1;
    cudaStream_t s = e->stream;
    ASDM_TRY(dalloc(&e->p, e->nparam, s));
    ASDM_TRY(dalloc(&e->g, e->nparam, s));
    ASDM_TRY(dalloc(&e->m, e->nparam, s));
    ASDM_TRY(dalloc(&e->v, e->nparam, s));
    ASDM_TRY(dalloc(&e->wb, 3 * asdm_estimator::kW, s));
    ASDM_TRY(dalloc(&e->err, 1, s));
    // Xavier-uniform weights from a seeded generator, zero biases
    std::vector<float> hp(e->nparam, 0.f);
    Rng rng(seed);
    const float a = std::sqrt(6.f / (kIn + kH));
    for (long long i = 0; i < 3 * asdm_estimator::kW; ++i) hp[i] = (float)((rng.uniform() * 2 - 1) * a);
    const float ao = std::sqrt(6.f / (kH + 1));
    for (int f = 0; f < kH; ++f) hp[3 * asdm_estimator::kW + 3 * kH + f] = (float)((rng.uniform() * 2 - 1) * ao);
    ASDM_CUDA(cudaMemcpyAsync(e->p, hp.data(), hp.size() * 4, cudaMemcpyHostToDevice, s));
    ASDM_CUDA(cudaMemsetAsync(e->m, 0, e->nparam * 4, s));
    ASDM_CUDA(cudaMemsetAsync(e->v, 0, e->nparam * 4, s));
    ASDM_CUDA(cudaMemsetAsync(e->err, 0, 4, s));
    to_bf16<<<grid_of(3 * asdm_estimator::kW), kT, 0, s>>>(e->p, e->wb, 3 * asdm_estimator::kW);
    ::asdm::count_launch();
    ASDM_CUDA(cudaStreamSynchronize(s));
    *out = e.release();
    return ASDM_OK;
}

extern "C" int asdm_est_predict(asdm_estimator *e, int n_nodes, int n_graphs, const float *x, const uint32_t *adj_off,
                                const uint32_t *adj, const uint32_t *node_graph, float *out) {
    clear_error();
    if (!e || !x || !adj_off || !node_graph || !out || n_nodes <= 0 || n_graphs <= 0)
        return fail(ASDM_ERR_INVALID, "bad estimator batch");
    ASDM_TRY(upload_batch(e, n_nodes, n_graphs, x, adj_off, adj, node_graph));
    ASDM_TRY(forward(e, n_nodes, n_graphs));
    ASDM_CUDA(cudaMemcpyAsync(out, e->y, (size_t)n_graphs * 4, cudaMemcpyDeviceToHost, e->stream));
    return check_err(e);
}

extern "C" int asdm_est_train_step(asdm_estimator *e, int n_nodes, int n_graphs, const float *x, const uint32_t *adj_off,
                                   const uint32_t *adj, const uint32_t *node_graph, const float *target, float lr,
                                   float *loss) {
    clear_error();
    if (!e || !x || !adj_off || !node_graph || !target || n_nodes <= 0 || n_graphs <= 0)
        return fail(ASDM_ERR_INVALID, "bad estimator batch");
    ASDM_TRY(upload_batch(e, n_nodes, n_graphs, x, adj_off, adj, node_graph));
    cudaStream_t s = e->stream;
    const int n = n_nodes, ng = n_graphs;
    const long long nh = (long long)n * kH;
    ASDM_CUDA(cudaMemcpyAsync(e->t, target, (size_t)ng * 4, cudaMemcpyHostToDevice, s));
    ASDM_TRY(forward(e, n, ng));
    ASDM_CUDA(cudaMemsetAsync(e->g, 0, e->nparam * 4, s));
    ASDM_CUDA(cudaMemsetAsync(e->loss, 0, 4, s));
    loss_grad<<<grid_of(ng), kT, 0, s>>>(e->y, e->t, e->gsum, e->wo(), ng, e->dy, e->loss, e->gwo(), e->gbo());
    readout_back<<<grid_of(nh), kT, 0, s>>>(e->dy, e->wo(), e->gid, n, e->dH);
    ::asdm::count_launch();
    ::asdm::count_launch();
    for (int l = kLayers - 1; l >= 0; --l) {
        float *Zl = e->Z + l * nh;
        __nv_bfloat16 *Xl = e->X + (long long)l * n * kIn;
        relu_back<<<grid_of(nh), kT, 0, s>>>(e->dH, Zl, n, e->dZ, e->gbias(l));
        ::asdm::count_launch();
        // dW_l[o][i] = sum_v dZ[v][o] X_l[v][i]   (M = 128 outputs, N = 256 inputs, K = nodes)
        tc::Operand a{e->dZ, 1, kH, kH};
        tc::Operand b{Xl, 1, kIn, kIn};
        ASDM_TRY(gemm(e, a, b, kH, kIn, n, e->gW(l), kIn, nullptr));
        if (l > 0) {
            // dX_l[v][i] = sum_o dZ[v][o] W_l[o][i]   (M = nodes, N = 256, K = 128)
            tc::Operand a2{e->dZ, kH, 1, n};
            tc::Operand b2{e->wb + l * asdm_estimator::kW, 1, kIn, kIn};
            ASDM_TRY(gemm(e, a2, b2, n, kIn, kH, e->dX, kIn, nullptr));
            x_back<<<grid_of(nh), kT, 0, s>>>(e->dX, e->adj_off, e->adj, n, e->dH);
            ::asdm::count_launch();
        }
    }
    e->step += 1;
    const float b1t = std::pow(0.9f, (float)e->step), b2t = std::pow(0.999f, (float)e->step);
    adam<<<grid_of(3 * asdm_estimator::kW), kT, 0, s>>>(e->p, e->g, e->m, e->v, 3 * asdm_estimator::kW, lr, b1t, b2t, e->wb);
    const long long rest = e->nparam - 3 * asdm_estimator::kW;
    adam<<<grid_of(rest), kT, 0, s>>>(e->p + 3 * asdm_estimator::kW, e->g + 3 * asdm_estimator::kW,
                                      e->m + 3 * asdm_estimator::kW, e->v + 3 * asdm_estimator::kW, rest, lr, b1t, b2t,
                                      nullptr);
    ::asdm::count_launch();
    ::asdm::count_launch();
    ASDM_CUDA(cudaGetLastError());
    if (loss) ASDM_CUDA(cudaMemcpyAsync(loss, e->loss, 4, cudaMemcpyDeviceToHost, s));
    return check_err(e);
}

extern "C" int asdm_est_params(asdm_estimator *e, float *out, uint64_t capacity, uint64_t *count) {
    if (!e) return fail(ASDM_ERR_INVALID, "null estimator");
    if (count) *count = (uint64_t)e->nparam;
    if (!out) return ASDM_OK;
    if (capacity < (uint64_t)e->nparam) return fail(ASDM_ERR_CAPACITY, "%lld parameters", e->nparam);
    ASDM_CUDA(cudaMemcpyAsync(out, e->p, e->nparam * 4, cudaMemcpyDeviceToHost, e->stream));
    ASDM_CUDA(cudaStreamSynchronize(e->stream));
    return ASDM_OK;
}

extern "C" int asdm_est_set_params(asdm_estimator *e, const float *in, uint64_t count) {
    if (!e || !in) return fail(ASDM_ERR_INVALID, "null argument");
    if (count != (uint64_t)e->nparam) return fail(ASDM_ERR_INVALID, "expected %lld parameters", e->nparam);
    ASDM_CUDA(cudaMemcpyAsync(e->p, in, e->nparam * 4, cudaMemcpyHostToDevice, e->stream));
    to_bf16<<<grid_of(3 * asdm_estimator::kW), kT, 0, e->stream>>>(e->p, e->wb, 3 * asdm_estimator::kW);
    ::asdm::count_launch();
    ASDM_CUDA(cudaStreamSynchronize(e->stream));
    return ASDM_OK;
}

extern "C" void asdm_est_free(asdm_estimator *e) {
    if (!e) return;
    free_batch(e);
    cudaStream_t s = e->stream;
    dfree(e->p, s); dfree(e->g, s); dfree(e->m, s); dfree(e->v, s); dfree(e->wb, s); dfree(e->err, s);
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    delete e;
}
