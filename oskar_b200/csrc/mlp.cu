// Multilayer perceptron with sine activations: training and inference
// kernels for the learned station-beam surrogate.
//
// Network: dims[0] -> dims[1] -> ... -> dims[L], L linear layers; every
// layer but the last is followed by sin(omega0 z) (the SIREN form, which
// represents the oscillatory array factor of a station far better than
// rectified or tanh units). Parameters live in one FP32 device array, per
// layer W [out][in] then b [out]; gradients and the Adam moments have the
// same layout.
//
// Kernels (all FP32, SIMT):
//  - gemm_kernel<TA, TB, EPI>: C[M][N] = op(A) op(B) over K in 64 x 64
//    tiles (16-deep k steps staged in shared memory, 4 x 4 outputs per
//    thread), with the epilogue fused: bias + sine (forward, keeping the
//    pre-activation for the backward pass), plain store (input gradient),
//    or atomic accumulation over batch slices (weight gradient);
//  - dz_kernel: dZ = dA omega0 cos(omega0 Z); bias_grad_kernel;
//  - mse_kernel (loss and its gradient), adam_kernel, gather_kernel
//    (minibatch rows by index).
// Training runs these per step; inference reuses the forward pass in
// chunks (no stored activations are kept beyond the chunk).
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "common.cuh"

namespace oskb {
namespace mlp {

constexpr int kT = 64;   // output tile edge
constexpr int kK = 16;   // k step
constexpr int kMaxLayers = 8;

enum Epi { kEpiForward = 0, kEpiStore = 1, kEpiAtomic = 2 };

struct GemmArgs
{
    int M, N, K;
    const float* A;  // op(A) is M x K
    const float* B;  // op(B) is K x N
    int lda, ldb;
    float* C;        // M x N, row-major, ld N
    float* Z;        // forward: pre-activation out (may be NULL)
    const float* bias;
    float omega0;
    int activate;
    int k_per_slice;  // atomic epilogue: K range per blockIdx.z
};

// op(A)[m][k] = TA ? A[k][m] : A[m][k]; op(B)[k][n] = TB ? B[n][k] : B[k][n]
template <bool TA, bool TB, int EPI>
__global__ void __launch_bounds__(256) gemm_kernel(const GemmArgs g)
{
    __shared__ float As[kK][kT + 4];
    __shared__ float Bs[kK][kT + 4];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int m0 = blockIdx.y * kT, n0 = blockIdx.x * kT;
    int k_begin = 0, k_end = g.K;
    if (EPI == kEpiAtomic)
    {
        k_begin = blockIdx.z * g.k_per_slice;
        k_end = min(g.K, k_begin + g.k_per_slice);
    }
    float acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
    for (int k0 = k_begin; k0 < k_end; k0 += kK)
    {
        for (int t = threadIdx.x; t < kK * kT; t += 256)
        {
            // A tile: As[kk][mm]; B tile: Bs[kk][nn]
            const int kk = TA ? t / kT : t % kK, mm = TA ? t % kT : t / kK;
            const int k = k0 + kk, m = m0 + mm;
            float a = 0.f;
            if (k < k_end && m < g.M)
                a = TA ? g.A[(size_t) k * g.lda + m] : g.A[(size_t) m * g.lda + k];
            As[kk][mm] = a;
            const int kb = TB ? t % kK : t / kT, nn = TB ? t / kK : t % kT;
            const int kq = k0 + kb, n = n0 + nn;
            float b = 0.f;
            if (kq < k_end && n < g.N)
                b = TB ? g.B[(size_t) n * g.ldb + kq] : g.B[(size_t) kq * g.ldb + n];
            Bs[kb][nn] = b;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kK; ++kk)
        {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            const int m = m0 + ty + 16 * i, n = n0 + tx + 16 * j;
            if (m >= g.M || n >= g.N) continue;
            const size_t o = (size_t) m * g.N + n;
            if (EPI == kEpiForward)
            {
                const float z = acc[i][j] + g.bias[n];
                if (g.Z) g.Z[o] = z;
                g.C[o] = g.activate ? sinf(g.omega0 * z) : z;
            }
            else if (EPI == kEpiStore)
                g.C[o] = acc[i][j];
            else
                atomicAdd(&g.C[o], acc[i][j]);
        }
}

// dZ = dA * omega0 * cos(omega0 Z), in place on dA.
__global__ void dz_kernel(long long n, float* __restrict__ dA,
        const float* __restrict__ Z, float omega0)
{
    const long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    if (i < n) dA[i] *= omega0 * cosf(omega0 * Z[i]);
}

// db[o] = sum_b dZ[b][o] (one warp per output, strided over the batch).
__global__ void bias_grad_kernel(int batch, int out,
        const float* __restrict__ dZ, float* __restrict__ db)
{
    const int o = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const int lane = threadIdx.x & 31;
    if (o >= out) return;
    float s = 0.f;
    for (int b = lane; b < batch; b += 32) s += dZ[(size_t) b * out + o];
    for (int d = 16; d > 0; d >>= 1) s += __shfl_xor_sync(0xffffffffu, s, d);
    if (lane == 0) db[o] = s;
}

// Mean squared error over n values: dy = 2 (y - t) / n; loss += sum / n.
// y and dy may be the same array (the gradient overwrites the outputs).
__global__ void mse_kernel(long long n, const float* y,
        const float* __restrict__ t, float* dy, float* __restrict__ loss)
{
    const long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    float e = 0.f;
    if (i < n)
    {
        const float d = y[i] - t[i];
        if (dy) dy[i] = 2.f * d / (float) n;
        e = d * d / (float) n;
    }
    for (int d = 16; d > 0; d >>= 1) e += __shfl_xor_sync(0xffffffffu, e, d);
    if ((threadIdx.x & 31) == 0 && loss) atomicAdd(loss, e);
}

__global__ void adam_kernel(int n, float* __restrict__ p,
        const float* __restrict__ g, float* __restrict__ m,
        float* __restrict__ v, float lr, float b1, float b2, float eps,
        float c1, float c2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// rows out[r][:] = in[idx[r]][:]
__global__ void gather_kernel(int rows, int cols, const int* __restrict__ idx,
        const float* __restrict__ in, float* __restrict__ out)
{
    const long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    if (i >= (long long) rows * cols) return;
    const int r = (int) (i / cols), c = (int) (i % cols);
    out[i] = in[(size_t) idx[r] * cols + c];
}

// Minibatch indices from a counter-based hash (splitmix64 of step, row).
__global__ void batch_index_kernel(int rows, int num_samples,
        unsigned long long seed, int step, int* __restrict__ idx)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    unsigned long long z = seed + 0x9E3779B97F4A7C15ULL *
            ((unsigned long long) step * 1000003ULL + r + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    idx[r] = (int) (z % (unsigned long long) num_samples);
}

int launch_gemm(bool ta, bool tb, int epi, GemmArgs g, int k_slices,
        cudaStream_t s)
{
    dim3 grid((g.N + kT - 1) / kT, (g.M + kT - 1) / kT,
            epi == kEpiAtomic ? k_slices : 1);
    if (epi == kEpiAtomic)
        g.k_per_slice = ((g.K + k_slices - 1) / k_slices + kK - 1) / kK * kK;
#define OSKB_G(A, B, E) gemm_kernel<A, B, E><<<grid, 256, 0, s>>>(g)
    if (epi == kEpiForward && !ta && tb) OSKB_G(false, true, kEpiForward);
    else if (epi == kEpiStore && !ta && !tb) OSKB_G(false, false, kEpiStore);
    else if (epi == kEpiAtomic && ta && !tb) OSKB_G(true, false, kEpiAtomic);
    else return OSKB_ERR_INVALID_ARGUMENT;
#undef OSKB_G
    return check_launch("mlp gemm");
}

}  // namespace mlp
}  // namespace oskb

struct oskb_Mlp
{
    int L;
    int dims[oskb::mlp::kMaxLayers + 1];
    float omega0;
    int num_params;
    int w_off[oskb::mlp::kMaxLayers], b_off[oskb::mlp::kMaxLayers];
    float *params, *grads, *m, *v;
    int max_batch, max_dim;
    float* act[oskb::mlp::kMaxLayers + 1];
    float* pre[oskb::mlp::kMaxLayers];
    float* dbuf[2];
    int* idx;
    float *xb, *tb, *yb, *loss;
    const float* last_x;
    int last_batch;
    int adam_step;
};

namespace {

using namespace oskb::mlp;

void free_work(oskb_Mlp* n)
{
    for (int l = 0; l <= kMaxLayers; ++l) { cudaFree(n->act[l]); n->act[l] = nullptr; }
    for (int l = 0; l < kMaxLayers; ++l) { cudaFree(n->pre[l]); n->pre[l] = nullptr; }
    cudaFree(n->dbuf[0]); cudaFree(n->dbuf[1]);
    cudaFree(n->idx); cudaFree(n->xb); cudaFree(n->tb); cudaFree(n->yb);
    n->dbuf[0] = n->dbuf[1] = nullptr;
    n->idx = nullptr; n->xb = n->tb = n->yb = nullptr;
    n->max_batch = 0;
}

int ensure_work(oskb_Mlp* n, int batch)
{
    if (batch <= n->max_batch) return 0;
    free_work(n);
    bool ok = true;
    const size_t b = (size_t) batch;
    for (int l = 1; l < n->L && ok; ++l)
        ok = cudaMalloc(&n->act[l], b * n->dims[l] * 4) == cudaSuccess &&
                cudaMalloc(&n->pre[l - 1], b * n->dims[l] * 4) == cudaSuccess;
    ok = ok && cudaMalloc(&n->dbuf[0], b * n->max_dim * 4) == cudaSuccess &&
            cudaMalloc(&n->dbuf[1], b * n->max_dim * 4) == cudaSuccess &&
            cudaMalloc(&n->idx, b * 4) == cudaSuccess &&
            cudaMalloc(&n->xb, b * n->dims[0] * 4) == cudaSuccess &&
            cudaMalloc(&n->tb, b * n->dims[n->L] * 4) == cudaSuccess &&
            cudaMalloc(&n->yb, b * n->dims[n->L] * 4) == cudaSuccess;
    if (!ok)
    {
        oskb::set_last_error("oskb_mlp workspace", cudaGetLastError());
        free_work(n);
        return OSKB_ERR_MEMORY_ALLOC_FAILURE;
    }
    n->max_batch = batch;
    return 0;
}

// Forward through all layers; keeps pre-activations when keep != 0.
int forward(oskb_Mlp* n, int batch, const float* x, float* y, bool keep,
        cudaStream_t s)
{
    const float* in = x;
    for (int l = 0; l < n->L; ++l)
    {
        const bool last = l == n->L - 1;
        GemmArgs g;
        memset(&g, 0, sizeof(g));
        g.M = batch; g.N = n->dims[l + 1]; g.K = n->dims[l];
        g.A = in; g.lda = n->dims[l];
        g.B = n->params + n->w_off[l]; g.ldb = n->dims[l];
        g.C = last ? y : n->act[l + 1];
        g.Z = (!last && keep) ? n->pre[l] : nullptr;
        g.bias = n->params + n->b_off[l];
        g.omega0 = n->omega0;
        g.activate = !last;
        if (int err = launch_gemm(false, true, kEpiForward, g, 1, s))
            return err;
        in = g.C;
    }
    return 0;
}

int backward(oskb_Mlp* n, int batch, const float* x, const float* dy,
        cudaStream_t s)
{
    cudaMemsetAsync(n->grads, 0, sizeof(float) * n->num_params, s);
    const int L = n->L;
    cudaMemcpyAsync(n->dbuf[0], dy, sizeof(float) * batch * n->dims[L],
            cudaMemcpyDeviceToDevice, s);
    int cur = 0;
    const int k_slices = max(1, min(64, batch / 256));
    for (int l = L - 1; l >= 0; --l)
    {
        const int in_dim = n->dims[l], out_dim = n->dims[l + 1];
        float* G = n->dbuf[cur];
        if (l < L - 1)
        {
            const long long cnt = (long long) batch * out_dim;
            dz_kernel<<<(unsigned) ((cnt + 255) / 256), 256, 0, s>>>(cnt, G,
                    n->pre[l], n->omega0);
        }
        const float* in = l == 0 ? x : n->act[l];
        GemmArgs g;
        memset(&g, 0, sizeof(g));
        g.M = out_dim; g.N = in_dim; g.K = batch;
        g.A = G; g.lda = out_dim;
        g.B = in; g.ldb = in_dim;
        g.C = n->grads + n->w_off[l];
        if (int err = launch_gemm(true, false, kEpiAtomic, g, k_slices, s))
            return err;
        bias_grad_kernel<<<(out_dim + 7) / 8, 256, 0, s>>>(batch, out_dim, G,
                n->grads + n->b_off[l]);
        if (l > 0)
        {
            GemmArgs h;
            memset(&h, 0, sizeof(h));
            h.M = batch; h.N = in_dim; h.K = out_dim;
            h.A = G; h.lda = out_dim;
            h.B = n->params + n->w_off[l]; h.ldb = in_dim;
            h.C = n->dbuf[cur ^ 1];
            if (int err = launch_gemm(false, false, kEpiStore, h, 1, s))
                return err;
            cur ^= 1;
        }
    }
    return oskb::check_launch("mlp backward");
}

double uniform01(unsigned long long& state)
{
    unsigned long long z = (state += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    return (z >> 11) * (1.0 / 9007199254740992.0);
}

}  // namespace

extern "C" {

void oskb_mlp_free(oskb_Mlp* n)
{
    if (!n) return;
    free_work(n);
    cudaFree(n->params); cudaFree(n->grads); cudaFree(n->m); cudaFree(n->v);
    cudaFree(n->loss);
    free(n);
}

oskb_Mlp* oskb_mlp_create(int num_layers, const int* dims, float omega0,
        unsigned long long seed, int* status)
{
    if (*status) return nullptr;
    if (num_layers < 1 || num_layers > kMaxLayers || !dims)
    {
        *status = OSKB_ERR_INVALID_ARGUMENT;
        return nullptr;
    }
    for (int l = 0; l <= num_layers; ++l)
        if (dims[l] < 1 || dims[l] > 4096)
        {
            *status = OSKB_ERR_INVALID_ARGUMENT;
            return nullptr;
        }
    oskb_Mlp* n = (oskb_Mlp*) calloc(1, sizeof(oskb_Mlp));
    n->L = num_layers;
    n->omega0 = omega0;
    int off = 0;
    for (int l = 0; l <= num_layers; ++l)
    {
        n->dims[l] = dims[l];
        n->max_dim = max(n->max_dim, dims[l]);
    }
    for (int l = 0; l < num_layers; ++l)
    {
        n->w_off[l] = off;
        off += dims[l] * dims[l + 1];
        n->b_off[l] = off;
        off += dims[l + 1];
    }
    n->num_params = off;
    // Sine-network initialisation: first layer U(-1/in, 1/in), later layers
    // U(-sqrt(6/in)/omega0, +sqrt(6/in)/omega0); biases U(-1/sqrt(in),
    // 1/sqrt(in)).
    std::vector<float> h(off);
    unsigned long long st = seed;
    for (int l = 0; l < num_layers; ++l)
    {
        const double in = dims[l];
        const double wb = l == 0 ? 1.0 / in : sqrt(6.0 / in) / omega0;
        const double bb = 1.0 / sqrt(in);
        for (int i = 0; i < dims[l] * dims[l + 1]; ++i)
            h[n->w_off[l] + i] = (float) ((2 * uniform01(st) - 1) * wb);
        for (int i = 0; i < dims[l + 1]; ++i)
            h[n->b_off[l] + i] = (float) ((2 * uniform01(st) - 1) * bb);
    }
    const size_t bytes = sizeof(float) * off;
    bool ok = cudaMalloc(&n->params, bytes) == cudaSuccess &&
            cudaMalloc(&n->grads, bytes) == cudaSuccess &&
            cudaMalloc(&n->m, bytes) == cudaSuccess &&
            cudaMalloc(&n->v, bytes) == cudaSuccess &&
            cudaMalloc(&n->loss, sizeof(float)) == cudaSuccess &&
            cudaMemcpy(n->params, h.data(), bytes, cudaMemcpyHostToDevice) ==
            cudaSuccess && cudaMemset(n->m, 0, bytes) == cudaSuccess &&
            cudaMemset(n->v, 0, bytes) == cudaSuccess &&
            cudaMemset(n->grads, 0, bytes) == cudaSuccess;
    if (!ok)
    {
        oskb::set_last_error("oskb_mlp_create", cudaGetLastError());
        oskb_mlp_free(n);
        *status = OSKB_ERR_MEMORY_ALLOC_FAILURE;
        return nullptr;
    }
    return n;
}

int oskb_mlp_num_params(const oskb_Mlp* n) { return n->num_params; }

int oskb_mlp_copy_to_host(const oskb_Mlp* n, int which, float* host)
{
    const float* src = which == 0 ? n->params : which == 1 ? n->grads :
            nullptr;
    if (!src || !host) return OSKB_ERR_INVALID_ARGUMENT;
    if (cudaMemcpy(host, src, sizeof(float) * n->num_params,
            cudaMemcpyDeviceToHost) != cudaSuccess)
    {
        oskb::set_last_error("oskb_mlp_copy_to_host", cudaGetLastError());
        return OSKB_ERR_MEMORY_COPY_FAILURE;
    }
    return 0;
}

int oskb_mlp_set_params(oskb_Mlp* n, const float* host)
{
    if (!host) return OSKB_ERR_INVALID_ARGUMENT;
    if (cudaMemcpy(n->params, host, sizeof(float) * n->num_params,
            cudaMemcpyHostToDevice) != cudaSuccess)
    {
        oskb::set_last_error("oskb_mlp_set_params", cudaGetLastError());
        return OSKB_ERR_MEMORY_COPY_FAILURE;
    }
    return 0;
}
float* oskb_mlp_params(oskb_Mlp* n) { return n->params; }
float* oskb_mlp_grads(oskb_Mlp* n) { return n->grads; }

int oskb_mlp_forward(oskb_Mlp* n, int batch, const float* x, float* y,
        void* stream)
{
    if (batch < 1 || !x || !y) return OSKB_ERR_INVALID_ARGUMENT;
    if (int err = ensure_work(n, batch)) return err;
    n->last_x = x;
    n->last_batch = batch;
    return forward(n, batch, x, y, true, oskb::as_stream(stream));
}

int oskb_mlp_backward(oskb_Mlp* n, int batch, const float* dy, void* stream)
{
    if (batch != n->last_batch || !n->last_x || !dy)
        return OSKB_ERR_INVALID_ARGUMENT;
    return backward(n, batch, n->last_x, dy, oskb::as_stream(stream));
}

int oskb_mlp_mse(long long count, const float* y, const float* target,
        float* dy, float* loss, void* stream)
{
    if (count < 1 || !y || !target) return OSKB_ERR_INVALID_ARGUMENT;
    mse_kernel<<<(unsigned) ((count + 255) / 256), 256, 0,
            oskb::as_stream(stream)>>>(count, y, target, dy, loss);
    return oskb::check_launch("oskb_mlp_mse");
}

int oskb_mlp_adam_step(oskb_Mlp* n, float lr, float beta1, float beta2,
        float eps, void* stream)
{
    ++n->adam_step;
    const float c1 = 1.f - powf(beta1, (float) n->adam_step);
    const float c2 = 1.f - powf(beta2, (float) n->adam_step);
    adam_kernel<<<(n->num_params + 255) / 256, 256, 0,
            oskb::as_stream(stream)>>>(n->num_params, n->params, n->grads,
            n->m, n->v, lr, beta1, beta2, eps, c1, c2);
    return oskb::check_launch("oskb_mlp_adam_step");
}

int oskb_mlp_train(oskb_Mlp* n, int num_samples, const float* x,
        const float* target, int batch, int steps, float lr_max,
        unsigned long long seed, int report_every, float* loss_history,
        void* stream)
{
    if (num_samples < 1 || batch < 1 || steps < 0 || !x || !target)
        return OSKB_ERR_INVALID_ARGUMENT;
    cudaStream_t s = oskb::as_stream(stream);
    if (int err = ensure_work(n, batch)) return err;
    const int din = n->dims[0], dout = n->dims[n->L];
    const long long cnt = (long long) batch * dout;
    for (int step = 0; step < steps; ++step)
    {
        batch_index_kernel<<<(batch + 255) / 256, 256, 0, s>>>(batch,
                num_samples, seed, step, n->idx);
        gather_kernel<<<(unsigned) (((long long) batch * din + 255) / 256),
                256, 0, s>>>(batch, din, n->idx, x, n->xb);
        gather_kernel<<<(unsigned) ((cnt + 255) / 256), 256, 0, s>>>(batch,
                dout, n->idx, target, n->tb);
        if (int err = forward(n, batch, n->xb, n->yb, true, s)) return err;
        const bool report = report_every > 0 && loss_history &&
                (step % report_every == 0 || step == steps - 1);
        if (report) cudaMemsetAsync(n->loss, 0, sizeof(float), s);
        // The loss gradient overwrites the outputs in place.
        mse_kernel<<<(unsigned) ((cnt + 255) / 256), 256, 0, s>>>(cnt, n->yb,
                n->tb, n->yb, report ? n->loss : nullptr);
        if (int err = backward(n, batch, n->xb, n->yb, s)) return err;
        const float lr = lr_max * 0.5f * (1.f + cosf(3.14159265f * step /
                (float) max(steps, 1)));
        if (int err = oskb_mlp_adam_step(n, lr, 0.9f, 0.999f, 1e-8f, s))
            return err;
        if (report)
        {
            float h = 0.f;
            cudaMemcpyAsync(&h, n->loss, sizeof(float),
                    cudaMemcpyDeviceToHost, s);
            if (cudaStreamSynchronize(s) != cudaSuccess)
            {
                oskb::set_last_error("oskb_mlp_train", cudaGetLastError());
                return OSKB_ERR_KERNEL_LAUNCH_FAILURE;
            }
            // slot k: step k * report_every; one more slot for the last
            // step when it is not a multiple of report_every.
            loss_history[step % report_every ? step / report_every + 1 :
                    step / report_every] = h;
        }
    }
    return oskb::check_launch("oskb_mlp_train");
}

int oskb_mlp_infer(oskb_Mlp* n, long long count, const float* x, float* y,
        int chunk, void* stream)
{
    if (count < 0 || (count && (!x || !y))) return OSKB_ERR_INVALID_ARGUMENT;
    if (chunk < 1) chunk = 65536;
    if (int err = ensure_work(n, chunk)) return err;
    cudaStream_t s = oskb::as_stream(stream);
    for (long long i = 0; i < count; i += chunk)
    {
        const int b = (int) (count - i < chunk ? count - i : chunk);
        if (int err = forward(n, b, x + i * n->dims[0], y + i * n->dims[n->L],
                false, s))
            return err;
    }
    return 0;
}

}  // extern "C"
