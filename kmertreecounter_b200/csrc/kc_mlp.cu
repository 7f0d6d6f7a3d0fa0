// Sizing model: a small MLP with BF16 weights and FP32 accumulation,
// trained and run by the project's own kernels.
//
//   x (4102 features) -> W1 + b1 -> ReLU -> W2 (512x512) + b2 -> ReLU
//   -> W3 (512x8192) + b3 -> y (log1p of predicted distinct keys and table keys
//   for 4096 buckets)
//
// All three layers and their gradients are one GEMM kernel on the tensor
// cores (mma.sync.m16n8k16 BF16 x BF16 -> FP32) with strided operands (so
// the transposed products of the backward pass need no copies) and fused
// epilogues (bias, ReLU, BF16 cast).  FP32 master weights and Adam state;
// BF16 copies feed the forward pass.  The network is ~6.6 M parameters and
// runs once per input file, far below the size at which tcgen05 tiles would
// change anything measurable.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../include/kmer_sizing.h"
#include "kc_internal.h"

namespace {

constexpr int GM = 64, GN = 64, GK = 32;  // CTA tile
constexpr int G_THREADS = 128;            // 4 warps, 2x2 of 32x32

enum Epi { EPI_STORE = 0, EPI_BIAS = 1, EPI_BIAS_RELU = 2 };

// C[m, n] = sum_k A[m, k] * B[k, n] (+ epilogue); element (i, j) of A at
// A[i*sa0 + j*sa1], of B at B[i*sb0 + j*sb1]; C row-major with ldc; optional
// BF16 copy of C.
struct GemmArgs {
    const __nv_bfloat16* A;
    const __nv_bfloat16* B;
    float* C;
    __nv_bfloat16* Cb;
    const float* bias;  // per column n
    int M, N, K;
    long sa0, sa1, sb0, sb1, ldc;
    int epi;
};

__device__ __forceinline__ uint32_t pack_bf16(__nv_bfloat16 lo, __nv_bfloat16 hi) {
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

__global__ void __launch_bounds__(G_THREADS) gemm_bf16(GemmArgs g) {
    __shared__ __nv_bfloat16 As[GM][GK + 8];  // [m][k]
    __shared__ __nv_bfloat16 Bs[GN][GK + 8];  // [n][k]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int m0 = blockIdx.y * GM, n0 = blockIdx.x * GN;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    const int grp = lane >> 2, tig = lane & 3;
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.f;
    const __nv_bfloat16 zero = __float2bfloat16(0.f);
    for (int k0 = 0; k0 < g.K; k0 += GK) {
        for (int e = tid; e < GM * GK; e += G_THREADS) {
            const int m = e / GK, k = e % GK;
            const long gm = m0 + m, gk = k0 + k;
            As[m][k] = (gm < g.M && gk < g.K) ? g.A[gm * g.sa0 + gk * g.sa1] : zero;
        }
        for (int e = tid; e < GN * GK; e += G_THREADS) {
            const int n = e / GK, k = e % GK;
            const long gn = n0 + n, gk = k0 + k;
            Bs[n][k] = (gn < g.N && gk < g.K) ? g.B[gk * g.sb0 + gn * g.sb1] : zero;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < GK; kk += 16) {
            uint32_t af[2][4], bf[4][2];
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const int r = wm + i * 16 + grp;
                const int c = kk + tig * 2;
                af[i][0] = pack_bf16(As[r][c], As[r][c + 1]);
                af[i][1] = pack_bf16(As[r + 8][c], As[r + 8][c + 1]);
                af[i][2] = pack_bf16(As[r][c + 8], As[r][c + 9]);
                af[i][3] = pack_bf16(As[r + 8][c + 8], As[r + 8][c + 9]);
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int n = wn + j * 8 + grp;
                const int c = kk + tig * 2;
                bf[j][0] = pack_bf16(Bs[n][c], Bs[n][c + 1]);
                bf[j][1] = pack_bf16(Bs[n][c + 8], Bs[n][c + 9]);
            }
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    asm volatile(
                        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
                        "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
                        : "+f"(acc[i][j][0]), "+f"(acc[i][j][1]), "+f"(acc[i][j][2]), "+f"(acc[i][j][3])
                        : "r"(af[i][0]), "r"(af[i][1]), "r"(af[i][2]), "r"(af[i][3]), "r"(bf[j][0]), "r"(bf[j][1]));
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int m = m0 + wm + i * 16 + grp + (r >= 2 ? 8 : 0);
                const int n = n0 + wn + j * 8 + tig * 2 + (r & 1);
                if (m >= g.M || n >= g.N) continue;
                float v = acc[i][j][r];
                if (g.epi == EPI_BIAS || g.epi == EPI_BIAS_RELU) v += g.bias[n];
                if (g.epi == EPI_BIAS_RELU) v = fmaxf(v, 0.f);
                g.C[(long)m * g.ldc + n] = v;
                if (g.Cb) g.Cb[(long)m * g.ldc + n] = __float2bfloat16(v);
            }
}

__global__ void to_bf16(const float* x, __nv_bfloat16* y, long n) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        y[i] = __float2bfloat16(x[i]);
}

// Weighted squared error w(e) e^2 with w = under for e < 0 (prediction below
// the target), 1 otherwise: dOut = 2 w e / n; loss = mean of w e^2.
__global__ void mse_grad(const float* out, const float* tgt, float* d, __nv_bfloat16* db, long n, float scale,
                         float under, float* loss) {
    float s = 0.f;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const float e = out[i] - tgt[i];
        const float w = e < 0.f ? under : 1.f;
        s += w * e * e;
        d[i] = 2.f * w * e * scale;
        db[i] = __float2bfloat16(d[i]);
    }
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, s * scale);
}

// dY *= (Y > 0), with a BF16 copy
__global__ void relu_back(float* d, const float* y, __nv_bfloat16* db, long n) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const float v = y[i] > 0.f ? d[i] : 0.f;
        d[i] = v;
        db[i] = __float2bfloat16(v);
    }
}

// bias gradient: column sums of d (rows x cols)
__global__ void col_sum(const float* d, float* g, int rows, int cols) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float s = 0.f;
    for (int r = 0; r < rows; ++r) s += d[(long)r * cols + c];
    g[c] = s;
}

// Adam on FP32 master weights, then the BF16 copy.
__global__ void adam(float* w, __nv_bfloat16* wb, const float* g, float* m, float* v, long n, float lr, float b1,
                     float b2, float eps, float c1, float c2) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        if (wb) wb[i] = __float2bfloat16(w[i]);
    }
}

thread_local std::string g_mlp_err;

}  // namespace

struct kc_mlp {
    int in, hid, out, max_batch;
    cudaStream_t st = nullptr;
    float *W[3] = {}, *b[3] = {}, *gW[3] = {}, *gb[3] = {}, *mW[3] = {}, *vW[3] = {}, *mb[3] = {}, *vb[3] = {};
    __nv_bfloat16* Wb[3] = {};
    long nW[3] = {}, nb[3] = {};
    float *x = nullptr, *h1 = nullptr, *h2 = nullptr, *y = nullptr, *t = nullptr;
    __nv_bfloat16 *xb = nullptr, *h1b = nullptr, *h2b = nullptr;
    float *dy = nullptr, *dh2 = nullptr, *dh1 = nullptr;
    __nv_bfloat16 *dyb = nullptr, *dh2b = nullptr, *dh1b = nullptr;
    float* loss = nullptr;
    float under = 1.f;  // loss weight of predictions below the target
    long step = 0;
};

namespace {

#define MK(x)                                                            \
    do {                                                                 \
        cudaError_t e_ = (x);                                            \
        if (e_ != cudaSuccess) {                                         \
            g_mlp_err = std::string(#x) + ": " + cudaGetErrorString(e_); \
            return KC_ERR_DEVICE;                                        \
        }                                                                \
    } while (0)

template <class T>
cudaError_t dalloc(T** p, long n) {
    return cudaMalloc(reinterpret_cast<void**>(p), std::max<long>(n, 1) * sizeof(T));
}

void gemm(cudaStream_t st, const __nv_bfloat16* A, long sa0, long sa1, const __nv_bfloat16* B, long sb0, long sb1,
          float* C, __nv_bfloat16* Cb, long ldc, const float* bias, int M, int N, int K, int epi) {
    GemmArgs g{A, B, C, Cb, bias, M, N, K, sa0, sa1, sb0, sb1, ldc, epi};
    dim3 grid((N + GN - 1) / GN, (M + GM - 1) / GM);
    gemm_bf16<<<grid, G_THREADS, 0, st>>>(g);
}

int forward(kc_mlp* m, int B) {
    const int I = m->in, H = m->hid, O = m->out;
    gemm(m->st, m->xb, I, 1, m->Wb[0], H, 1, m->h1, m->h1b, H, m->b[0], B, H, I, EPI_BIAS_RELU);
    gemm(m->st, m->h1b, H, 1, m->Wb[1], H, 1, m->h2, m->h2b, H, m->b[1], B, H, H, EPI_BIAS_RELU);
    gemm(m->st, m->h2b, H, 1, m->Wb[2], O, 1, m->y, nullptr, O, m->b[2], B, O, H, EPI_BIAS);
    MK(cudaGetLastError());
    return KC_OK;
}

int backward(kc_mlp* m, int B, float* h_loss) {
    const int I = m->in, H = m->hid, O = m->out;
    const long nout = (long)B * O;
    MK(cudaMemsetAsync(m->loss, 0, sizeof(float), m->st));
    mse_grad<<<256, 256, 0, m->st>>>(m->y, m->t, m->dy, m->dyb, nout, 1.f / (float)nout, m->under, m->loss);
    // layer 3: gW3 = h2^T dy, gb3 = colsum(dy), dh2 = dy W3^T
    gemm(m->st, m->h2b, 1, H, m->dyb, O, 1, m->gW[2], nullptr, O, nullptr, H, O, B, EPI_STORE);
    col_sum<<<(O + 255) / 256, 256, 0, m->st>>>(m->dy, m->gb[2], B, O);
    gemm(m->st, m->dyb, O, 1, m->Wb[2], 1, O, m->dh2, nullptr, H, nullptr, B, H, O, EPI_STORE);
    relu_back<<<256, 256, 0, m->st>>>(m->dh2, m->h2, m->dh2b, (long)B * H);
    // layer 2
    gemm(m->st, m->h1b, 1, H, m->dh2b, H, 1, m->gW[1], nullptr, H, nullptr, H, H, B, EPI_STORE);
    col_sum<<<(H + 255) / 256, 256, 0, m->st>>>(m->dh2, m->gb[1], B, H);
    gemm(m->st, m->dh2b, H, 1, m->Wb[1], 1, H, m->dh1, nullptr, H, nullptr, B, H, H, EPI_STORE);
    relu_back<<<256, 256, 0, m->st>>>(m->dh1, m->h1, m->dh1b, (long)B * H);
    // layer 1
    gemm(m->st, m->xb, 1, I, m->dh1b, H, 1, m->gW[0], nullptr, H, nullptr, I, H, B, EPI_STORE);
    col_sum<<<(H + 255) / 256, 256, 0, m->st>>>(m->dh1, m->gb[0], B, H);
    MK(cudaGetLastError());
    if (h_loss) {
        MK(cudaMemcpyAsync(h_loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->st));
        MK(cudaStreamSynchronize(m->st));
    }
    return KC_OK;
}

int load_batch(kc_mlp* m, const float* x, const float* t, int B) {
    if (B < 1 || B > m->max_batch) {
        g_mlp_err = "batch size out of range";
        return KC_ERR_INVALID;
    }
    MK(cudaMemcpyAsync(m->x, x, (size_t)B * m->in * sizeof(float), cudaMemcpyHostToDevice, m->st));
    to_bf16<<<256, 256, 0, m->st>>>(m->x, m->xb, (long)B * m->in);
    if (t) MK(cudaMemcpyAsync(m->t, t, (size_t)B * m->out * sizeof(float), cudaMemcpyHostToDevice, m->st));
    MK(cudaGetLastError());
    return KC_OK;
}

}  // namespace

extern "C" {

const char* kc_mlp_last_error(void) { return g_mlp_err.c_str(); }

void kc_mlp_destroy(kc_mlp* m) {
    if (!m) return;
    if (m->st) cudaStreamSynchronize(m->st);
    for (int l = 0; l < 3; ++l)
        for (void* p : {(void*)m->W[l], (void*)m->Wb[l], (void*)m->gW[l], (void*)m->mW[l], (void*)m->vW[l],
                        (void*)m->b[l], (void*)m->gb[l], (void*)m->mb[l], (void*)m->vb[l]})
            if (p) cudaFree(p);
    for (void* p : {(void*)m->x, (void*)m->xb, (void*)m->h1, (void*)m->h1b, (void*)m->h2, (void*)m->h2b, (void*)m->y,
                    (void*)m->t, (void*)m->dy, (void*)m->dyb, (void*)m->dh2, (void*)m->dh2b, (void*)m->dh1,
                    (void*)m->dh1b, (void*)m->loss})
        if (p) cudaFree(p);
    if (m->st) cudaStreamDestroy(m->st);
    delete m;
}

// Replace layer l's weights (row-major fan_in x fan_out) and bias; resets the
// Adam state of that layer.
int kc_mlp_set_layer(kc_mlp* m, int l, const float* w, const float* bias) {
    if (!m || l < 0 || l > 2 || !w || !bias) return KC_ERR_INVALID;
    MK(cudaMemcpyAsync(m->W[l], w, m->nW[l] * sizeof(float), cudaMemcpyHostToDevice, m->st));
    MK(cudaMemcpyAsync(m->b[l], bias, m->nb[l] * sizeof(float), cudaMemcpyHostToDevice, m->st));
    to_bf16<<<256, 256, 0, m->st>>>(m->W[l], m->Wb[l], m->nW[l]);
    MK(cudaMemsetAsync(m->mW[l], 0, m->nW[l] * sizeof(float), m->st));
    MK(cudaMemsetAsync(m->vW[l], 0, m->nW[l] * sizeof(float), m->st));
    MK(cudaMemsetAsync(m->mb[l], 0, m->nb[l] * sizeof(float), m->st));
    MK(cudaMemsetAsync(m->vb[l], 0, m->nb[l] * sizeof(float), m->st));
    MK(cudaStreamSynchronize(m->st));
    m->step = 0;
    return KC_OK;
}

int kc_mlp_create(int in, int hid, int out, int max_batch, uint64_t seed, kc_mlp** res) {
    if (!res || in < 1 || hid < 1 || out < 1 || max_batch < 1) return KC_ERR_INVALID;
    *res = nullptr;
    kc_mlp* m = new kc_mlp();
    m->in = in;
    m->hid = hid;
    m->out = out;
    m->max_batch = max_batch;
    const int dims[4] = {in, hid, hid, out};
    // the network's kernels at the device's highest priority: a prediction
    // made beside a count is not held up by the count's queued kernels
    int prio_low = 0, prio_high = 0;
    cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
    if (cudaStreamCreateWithPriority(&m->st, cudaStreamNonBlocking, prio_high) != cudaSuccess) {
        delete m;
        g_mlp_err = "stream creation failed";
        return KC_ERR_DEVICE;
    }
    bool ok = true;
    for (int l = 0; l < 3; ++l) {
        m->nW[l] = (long)dims[l] * dims[l + 1];
        m->nb[l] = dims[l + 1];
        ok &= dalloc(&m->W[l], m->nW[l]) == cudaSuccess && dalloc(&m->Wb[l], m->nW[l]) == cudaSuccess &&
              dalloc(&m->gW[l], m->nW[l]) == cudaSuccess && dalloc(&m->mW[l], m->nW[l]) == cudaSuccess &&
              dalloc(&m->vW[l], m->nW[l]) == cudaSuccess && dalloc(&m->b[l], m->nb[l]) == cudaSuccess &&
              dalloc(&m->gb[l], m->nb[l]) == cudaSuccess && dalloc(&m->mb[l], m->nb[l]) == cudaSuccess &&
              dalloc(&m->vb[l], m->nb[l]) == cudaSuccess;
    }
    const long B = max_batch;
    ok &= dalloc(&m->x, B * in) == cudaSuccess && dalloc(&m->xb, B * in) == cudaSuccess &&
          dalloc(&m->h1, B * hid) == cudaSuccess && dalloc(&m->h1b, B * hid) == cudaSuccess &&
          dalloc(&m->h2, B * hid) == cudaSuccess && dalloc(&m->h2b, B * hid) == cudaSuccess &&
          dalloc(&m->y, B * out) == cudaSuccess && dalloc(&m->t, B * out) == cudaSuccess &&
          dalloc(&m->dy, B * out) == cudaSuccess && dalloc(&m->dyb, B * out) == cudaSuccess &&
          dalloc(&m->dh2, B * hid) == cudaSuccess && dalloc(&m->dh2b, B * hid) == cudaSuccess &&
          dalloc(&m->dh1, B * hid) == cudaSuccess && dalloc(&m->dh1b, B * hid) == cudaSuccess &&
          dalloc(&m->loss, 1) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        g_mlp_err = "device allocation failed";
        kc_mlp_destroy(m);
        return KC_ERR_NOMEM;
    }
    // He initialisation from a seeded xorshift generator (Box-Muller), zero biases
    uint64_t s = seed ? seed : 1;
    auto rnd = [&]() {
        s ^= s << 13;
        s ^= s >> 7;
        s ^= s << 17;
        return (double)(s >> 11) * (1.0 / 9007199254740992.0);
    };
    for (int l = 0; l < 3; ++l) {
        std::vector<float> w(m->nW[l]);
        const double sd = std::sqrt(2.0 / dims[l]) * (l == 2 ? 0.1 : 1.0);
        for (auto& v : w) {
            const double u1 = std::max(rnd(), 1e-12), u2 = rnd();
            v = (float)(sd * std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2));
        }
        std::vector<float> z(m->nb[l], 0.f);
        const int rc = kc_mlp_set_layer(m, l, w.data(), z.data());
        if (rc) {
            kc_mlp_destroy(m);
            return rc;
        }
    }
    *res = m;
    return KC_OK;
}

int kc_mlp_set_under_weight(kc_mlp* m, float under) {
    if (!m || !(under > 0.f)) return KC_ERR_INVALID;
    m->under = under;
    return KC_OK;
}

int kc_mlp_get_layer(kc_mlp* m, int l, float* w, float* bias) {
    if (!m || l < 0 || l > 2) return KC_ERR_INVALID;
    if (w) MK(cudaMemcpyAsync(w, m->W[l], m->nW[l] * sizeof(float), cudaMemcpyDeviceToHost, m->st));
    if (bias) MK(cudaMemcpyAsync(bias, m->b[l], m->nb[l] * sizeof(float), cudaMemcpyDeviceToHost, m->st));
    MK(cudaStreamSynchronize(m->st));
    return KC_OK;
}

int kc_mlp_forward(kc_mlp* m, const float* x, int B, float* y) {
    if (!m || !x || !y) return KC_ERR_INVALID;
    int rc = load_batch(m, x, nullptr, B);
    if (rc || (rc = forward(m, B))) return rc;
    MK(cudaMemcpyAsync(y, m->y, (size_t)B * m->out * sizeof(float), cudaMemcpyDeviceToHost, m->st));
    MK(cudaStreamSynchronize(m->st));
    return KC_OK;
}

int kc_mlp_gradients(kc_mlp* m, const float* x, const float* t, int B, int l, float* gw, float* gbias, float* loss) {
    if (!m || !x || !t || l < 0 || l > 2) return KC_ERR_INVALID;
    int rc = load_batch(m, x, t, B);
    if (rc || (rc = forward(m, B)) || (rc = backward(m, B, loss))) return rc;
    if (gw) MK(cudaMemcpyAsync(gw, m->gW[l], m->nW[l] * sizeof(float), cudaMemcpyDeviceToHost, m->st));
    if (gbias) MK(cudaMemcpyAsync(gbias, m->gb[l], m->nb[l] * sizeof(float), cudaMemcpyDeviceToHost, m->st));
    MK(cudaStreamSynchronize(m->st));
    return KC_OK;
}

int kc_mlp_train_step(kc_mlp* m, const float* x, const float* t, int B, float lr, float* loss) {
    if (!m || !x || !t) return KC_ERR_INVALID;
    int rc = load_batch(m, x, t, B);
    if (rc || (rc = forward(m, B)) || (rc = backward(m, B, loss))) return rc;
    m->step++;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float c1 = 1.f - std::pow(b1, (float)m->step), c2 = 1.f - std::pow(b2, (float)m->step);
    for (int l = 0; l < 3; ++l) {
        adam<<<512, 256, 0, m->st>>>(m->W[l], m->Wb[l], m->gW[l], m->mW[l], m->vW[l], m->nW[l], lr, b1, b2, eps, c1,
                                     c2);
        adam<<<64, 256, 0, m->st>>>(m->b[l], nullptr, m->gb[l], m->mb[l], m->vb[l], m->nb[l], lr, b1, b2, eps, c1, c2);
    }
    MK(cudaGetLastError());
    return KC_OK;
}

}  // extern "C"
