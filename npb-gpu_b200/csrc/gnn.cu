// gnn.cu -- the learned preconditioner: a message-passing network over the
// sparsity graph of A that emits a lower-triangular factor G on A's lower
// pattern, so that M = G^T G is SPD by construction.  Hand-written CUDA
// forward, backward (training) and inference kernels, all FP32, plus Adam.
// No counterpart in the reference; the network and its loss are defined in
// oracle/gnn_oracle.py's docstring, which the tests check these kernels
// against.
//
// Layout: every node matrix (features, hidden states, probe blocks) is
// n x 32 row-major, so one warp owns one row and lane c holds column c --
// the products with the sparse matrices are warp-per-row SpMMs with one
// 128-byte gather per stored entry.  Reductions over rows (weight gradients,
// loss terms) go through per-CTA partials summed in a fixed order, so a
// training step is deterministic.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "cgb_internal.h"

namespace cgb {
namespace gnn {

constexpr int kH = 32;     // hidden width
constexpr int kF = 4;      // input features
constexpr int kL = 3;      // message-passing layers
constexpr int kK = 32;     // probe vectors per training step
constexpr int kRedBlocks = 256;  // CTAs of the row reductions

// Offsets of the flat parameter vector (see oracle/gnn_oracle.py).
constexpr int kOffWin = 0;
constexpr int kOffBin = kOffWin + kF * kH;
constexpr int kOffLayer = kOffBin + kH;                 // + l * kLayerSize
constexpr int kLayerSize = 2 * kH * kH + kH;           // Ws, Wm, b
constexpr int kOffWd = kOffLayer + kL * kLayerSize;
constexpr int kOffCd = kOffWd + kH;
constexpr int kOffWe = kOffCd + 1;
constexpr int kOffCe = kOffWe + kH;
constexpr int kNumParams = kOffCe + 1;

__device__ __forceinline__ float warp_sum_f(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ float softplus_f(float u) { return u > 20.f ? u : log1pf(expf(u)); }
__device__ __forceinline__ float sigmoid_f(float u) { return 1.f / (1.f + expf(-u)); }

// ----------------------------------------------------------------- forward
// out[i,:] = act(in[i,:in_dim] W + b (+ add[i,:])), W in_dim x 32 row-major.
__global__ void k_dense(const float *__restrict__ in, int in_dim, const float *__restrict__ W,
                        const float *__restrict__ b, const float *__restrict__ add, float *out,
                        int n, int relu)
{
    __shared__ float sW[kH * kH];
    for (int t = threadIdx.x; t < in_dim * kH; t += blockDim.x) sW[t] = W[t];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const float bc = b ? b[lane] : 0.f;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n;
         i += (gridDim.x * blockDim.x) >> 5) {
        const float xi = lane < in_dim ? in[size_t(i) * in_dim + lane] : 0.f;
        float acc = bc;
        for (int k = 0; k < in_dim; k++) acc = fmaf(__shfl_sync(0xffffffffu, xi, k), sW[k * kH + lane], acc);
        if (add) acc += add[size_t(i) * kH + lane];
        out[size_t(i) * kH + lane] = relu ? fmaxf(acc, 0.f) : acc;
    }
}

// out[i,:] = in1[i,:] W1^T + in2[i,:] W2^T (both 32 x 32; in2/W2 optional).
__global__ void k_dense_t2(const float *__restrict__ in1, const float *__restrict__ W1,
                           const float *__restrict__ in2, const float *__restrict__ W2, float *out,
                           int n)
{
    __shared__ float s1[kH * kH], s2[kH * kH];
    for (int t = threadIdx.x; t < kH * kH; t += blockDim.x) {
        s1[t] = W1[t];
        s2[t] = W2 ? W2[t] : 0.f;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n;
         i += (gridDim.x * blockDim.x) >> 5) {
        const float a1 = in1[size_t(i) * kH + lane];
        const float a2 = in2 ? in2[size_t(i) * kH + lane] : 0.f;
        float acc = 0.f;
        for (int k = 0; k < kH; k++) {
            acc = fmaf(__shfl_sync(0xffffffffu, a1, k), s1[lane * kH + k], acc);
            if (in2) acc = fmaf(__shfl_sync(0xffffffffu, a2, k), s2[lane * kH + k], acc);
        }
        out[size_t(i) * kH + lane] = acc;
    }
}

// out[i,:] = dscale*in[i,:] + sum_k w_k in[col_k,:], w_k = val[k] or
// val[map[k]] (map may be null); diag may be null (then the row's own term
// is diag_const * in[i,:]).
__global__ void k_spmm(const int *__restrict__ ptr, const int *__restrict__ col,
                       const float *__restrict__ val, const int *__restrict__ map,
                       const float *__restrict__ diag, float diag_const,
                       const float *__restrict__ in, float *out, int n)
{
    const int lane = threadIdx.x & 31;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n;
         i += (gridDim.x * blockDim.x) >> 5) {
        const float d = diag ? diag[i] : diag_const;
        float acc = d * in[size_t(i) * kH + lane];
        const int k0 = ptr[i], k1 = ptr[i + 1];
        int k = k0;
        for (; k + 4 <= k1; k += 4) {
            float w[4], x[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                w[u] = map ? val[map[k + u]] : val[k + u];
                x[u] = in[size_t(col[k + u]) * kH + lane];
            }
#pragma unroll
            for (int u = 0; u < 4; u++) acc = fmaf(w[u], x[u], acc);
        }
        for (; k < k1; k++) acc = fmaf(map ? val[map[k]] : val[k], in[size_t(col[k]) * kH + lane], acc);
        out[size_t(i) * kH + lane] = acc;
    }
}

// Output head: g_ii = softplus(h_i.w_d + c_d); g_ij = ahat_ij (sum_c w_e h_i h_j + c_e).
__global__ void k_head(const float *__restrict__ h, const int *__restrict__ lptr,
                       const int *__restrict__ lcol, const float *__restrict__ lval,
                       const float *__restrict__ P, float *goff, float *gdiag, float *ud, int n)
{
    const int lane = threadIdx.x & 31;
    const float we = P[kOffWe + lane], wd = P[kOffWd + lane], ce = P[kOffCe], cd = P[kOffCd];
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n;
         i += (gridDim.x * blockDim.x) >> 5) {
        const float hi = h[size_t(i) * kH + lane];
        const float u = warp_sum_f(hi * wd) + cd;
        if (lane == 0) {
            ud[i] = u;
            gdiag[i] = softplus_f(u);
        }
        const float hw = hi * we;
        for (int k = lptr[i]; k < lptr[i + 1]; k++) {
            const float v = warp_sum_f(hw * h[size_t(lcol[k]) * kH + lane]) + ce;
            if (lane == 0) goff[k] = lval[k] * v;
        }
    }
}

// ------------------------------------------------------------ reductions
// part[blk][c] = sum over this CTA's rows of a[i,c]*b[i,c] (b null: a^2).
__global__ void k_colsum_prod(const float *__restrict__ a, const float *__restrict__ b, int n,
                              float *part)
{
    __shared__ float s[32][33];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float acc = 0.f;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n;
         i += (gridDim.x * blockDim.x) >> 5) {
        const float x = a[size_t(i) * kH + lane];
        acc = fmaf(x, b ? b[size_t(i) * kH + lane] : x, acc);
    }
    s[warp][lane] = acc;
    __syncthreads();
    if (warp == 0) {
        float t = 0.f;
        for (int w = 0; w < int(blockDim.x >> 5); w++) t += s[w][lane];
        part[blockIdx.x * kH + lane] = t;
    }
}

// part[blk][k*32 + c] = sum over this CTA's rows of a[i,k] * b[i,c]
// (a: n x ka, ka <= 32) and part[blk][ka*32 + c] = sum b[i,c].
__global__ void k_outer(const float *__restrict__ a, int ka, const float *__restrict__ b, int n,
                        float *part)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float acc[kH + 1];
#pragma unroll
    for (int k = 0; k <= kH; k++) acc[k] = 0.f;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n;
         i += (gridDim.x * blockDim.x) >> 5) {
        const float ai = lane < ka ? a[size_t(i) * ka + lane] : 0.f;
        const float bi = b[size_t(i) * kH + lane];
#pragma unroll
        for (int k = 0; k < kH; k++) acc[k] = fmaf(__shfl_sync(0xffffffffu, ai, k), bi, acc[k]);
        acc[kH] += bi;
    }
    __shared__ float s[8][kH + 1][kH];  // up to 8 warps
#pragma unroll
    for (int k = 0; k <= kH; k++) s[warp][k][lane] = acc[k];
    __syncthreads();
    for (int t = threadIdx.x; t < (kH + 1) * kH; t += blockDim.x) {
        const int k = t / kH, c = t % kH;
        if (k < ka || k == kH) {
            float v = 0.f;
            for (int w = 0; w < int(blockDim.x >> 5); w++) v += s[w][k][c];
            part[size_t(blockIdx.x) * (kH + 1) * kH + t] = v;
        }
    }
}

// out[t] = sum_blk part[blk][t] for t < count (fixed order); optional add-to.
__global__ void k_reduce_parts(const float *__restrict__ part, int nparts, int stride, int count,
                               float *out, int accumulate)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x) {
        float v = 0.f;
        for (int p = 0; p < nparts; p++) v += part[size_t(p) * stride + t];
        out[t] = accumulate ? out[t] + v : v;
    }
}

// --------------------------------------------------------- loss / probes
// out[i,c] = scale[c] * (a[i,c] - b[i,c])  (b optional), scale optional.
__global__ void k_axpy_cols(const float *__restrict__ a, const float *__restrict__ b,
                            const float *__restrict__ scale, float *out, int n)
{
    const size_t total = size_t(n) * kH;
    for (size_t t = blockIdx.x * size_t(blockDim.x) + threadIdx.x; t < total;
         t += size_t(gridDim.x) * blockDim.x) {
        const int c = int(t % kH);
        float v = a[t] - (b ? b[t] : 0.f);
        if (scale) v *= scale[c];
        out[t] = v;
    }
}

// dG on the lower pattern: dGoff[e] = sum_k T[i,k] GU[j,k] + GT[i,k] R[j,k];
// dGdiag[i] the same with j = i.
__global__ void k_dG(const float *__restrict__ T, const float *__restrict__ GU,
                     const float *__restrict__ GT, const float *__restrict__ R,
                     const int *__restrict__ lptr, const int *__restrict__ lcol, float *dGoff,
                     float *dGdiag, int n)
{
    const int lane = threadIdx.x & 31;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n;
         i += (gridDim.x * blockDim.x) >> 5) {
        const float ti = T[size_t(i) * kH + lane], gti = GT[size_t(i) * kH + lane];
        const float dd = warp_sum_f(ti * GU[size_t(i) * kH + lane] + gti * R[size_t(i) * kH + lane]);
        if (lane == 0) dGdiag[i] = dd;
        for (int k = lptr[i]; k < lptr[i + 1]; k++) {
            const size_t j = size_t(lcol[k]) * kH + lane;
            const float v = warp_sum_f(ti * GU[j] + gti * R[j]);
            if (lane == 0) dGoff[k] = v;
        }
    }
}

// Head backward, pass 1 (rows i over their lower entries): dh_i, dv, and per
// CTA partials of dw_e (32), dc_e, dw_d (32), dc_d.
__global__ void k_head_bwd_rows(const float *__restrict__ h, const int *__restrict__ lptr,
                                const int *__restrict__ lcol, const float *__restrict__ lval,
                                const float *__restrict__ P, const float *__restrict__ dGoff,
                                const float *__restrict__ dGdiag, const float *__restrict__ ud,
                                float *dv, float *dh, float *part, int n)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const float we = P[kOffWe + lane], wd = P[kOffWd + lane];
    float awe = 0.f, ace = 0.f, awd = 0.f, acd = 0.f;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n;
         i += (gridDim.x * blockDim.x) >> 5) {
        const float hi = h[size_t(i) * kH + lane];
        const float du = dGdiag[i] * sigmoid_f(ud[i]);
        float dhi = du * wd;
        awd = fmaf(du, hi, awd);
        acd += (lane == 0) ? du : 0.f;
        for (int k = lptr[i]; k < lptr[i + 1]; k++) {
            const float d = dGoff[k] * lval[k];
            const float hj = h[size_t(lcol[k]) * kH + lane];
            dhi = fmaf(d * we, hj, dhi);
            awe = fmaf(d, hi * hj, awe);
            ace += (lane == 0) ? d : 0.f;
            if (lane == 0) dv[k] = d;
        }
        dh[size_t(i) * kH + lane] = dhi;
    }
    __shared__ float s[8][66];
    s[warp][lane] = awe;
    s[warp][32 + lane] = awd;
    if (lane == 0) {
        s[warp][64] = ace;
        s[warp][65] = acd;
    }
    __syncthreads();
    for (int t = threadIdx.x; t < 66; t += blockDim.x) {
        float v = 0.f;
        for (int w = 0; w < int(blockDim.x >> 5); w++) v += s[w][t];
        part[blockIdx.x * 66 + t] = v;
    }
}

// Head backward, pass 2 (rows j over the transposed lower pattern): adds
// sum_{i>j} dv_ij w_e h_i into dh_j.
__global__ void k_head_bwd_cols(const float *__restrict__ h, const int *__restrict__ uptr,
                                const int *__restrict__ urow, const int *__restrict__ umap,
                                const float *__restrict__ P, const float *__restrict__ dv,
                                float *dh, int n)
{
    const int lane = threadIdx.x & 31;
    const float we = P[kOffWe + lane];
    for (int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < n;
         j += (gridDim.x * blockDim.x) >> 5) {
        float acc = dh[size_t(j) * kH + lane];
        for (int k = uptr[j]; k < uptr[j + 1]; k++)
            acc = fmaf(dv[umap[k]] * we, h[size_t(urow[k]) * kH + lane], acc);
        dh[size_t(j) * kH + lane] = acc;
    }
}

// dz = dh * (h > 0)
__global__ void k_relu_bwd(const float *__restrict__ dh, const float *__restrict__ h, float *dz,
                           size_t total)
{
    for (size_t t = blockIdx.x * size_t(blockDim.x) + threadIdx.x; t < total;
         t += size_t(gridDim.x) * blockDim.x)
        dz[t] = h[t] > 0.f ? dh[t] : 0.f;
}

// Adam on the flat parameter vector.
__global__ void k_adam(float *P, const float *__restrict__ g, float *m, float *v, int count,
                       float lr, float b1, float b2, float eps, float c1, float c2)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x) {
        const float gt = g[t];
        const float mt = b1 * m[t] + (1.f - b1) * gt;
        const float vt = b2 * v[t] + (1.f - b2) * gt * gt;
        m[t] = mt;
        v[t] = vt;
        P[t] -= lr * (mt / c1) / (sqrtf(vt / c2) + eps);
    }
}

// Counter-based normal variates for the random probes.
__device__ __forceinline__ unsigned hash_u32(unsigned x)
{
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

__global__ void k_normal(float *out, size_t total, unsigned seed)
{
    for (size_t t = blockIdx.x * size_t(blockDim.x) + threadIdx.x; t < total;
         t += size_t(gridDim.x) * blockDim.x) {
        const unsigned a = hash_u32(unsigned(t) * 2u + 1u + seed * 0x9e3779b9u);
        const unsigned b = hash_u32(unsigned(t) * 2u + 2u + seed * 0x85ebca6bu);
        const float u1 = (float(a >> 8) + 1.f) * (1.f / 16777217.f);
        const float u2 = float(b >> 8) * (1.f / 16777216.f);
        out[t] = sqrtf(-2.f * logf(u1)) * cospif(2.f * u2);
    }
}

// Batched CG step on Ahat for 32 right-hand sides (columns), per column
// coefficients: x += alpha p, r -= alpha q (x optional).
__global__ void k_cg_update(float *r, const float *__restrict__ q, const float *__restrict__ alpha,
                            int n)
{
    const size_t total = size_t(n) * kH;
    for (size_t t = blockIdx.x * size_t(blockDim.x) + threadIdx.x; t < total;
         t += size_t(gridDim.x) * blockDim.x)
        r[t] -= alpha[t % kH] * q[t];
}

__global__ void k_cg_dir(float *p, const float *__restrict__ r, const float *__restrict__ beta, int n)
{
    const size_t total = size_t(n) * kH;
    for (size_t t = blockIdx.x * size_t(blockDim.x) + threadIdx.x; t < total;
         t += size_t(gridDim.x) * blockDim.x)
        p[t] = r[t] + beta[t % kH] * p[t];
}

// Per-column coefficient: out[c] = num[c] / den[c] (0 if den is 0); with
// `keep` the numerator is also copied to prev[c] (CG's rho bookkeeping).
__global__ void k_ratio(const float *__restrict__ num, const float *__restrict__ den, float *out)
{
    const int c = threadIdx.x;
    if (c < kH) out[c] = den[c] != 0.f ? num[c] / den[c] : 0.f;
}

// Loss-side coefficient: s[c] = (2/K) / |r_c|^2, and L = (1/K) sum_c |w_c|^2 / |r_c|^2.
__global__ void k_loss_coef(const float *__restrict__ rn2, const float *__restrict__ wn2, float *s,
                            float *loss)
{
    const int c = threadIdx.x;
    float l = 0.f;
    if (c < kH) {
        s[c] = (2.f / kK) / rn2[c];
        l = wn2[c] / rn2[c] / kK;
    }
    l = warp_sum_f(l);
    if (c == 0) *loss = l;
}

}  // namespace gnn
}  // namespace cgb

// ===================================================================== host
using namespace cgb;
using namespace cgb::gnn;

#define GNN_TRY(call)                                                                     \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return set_error(CGB_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                             __FILE__, __LINE__);                                         \
    } while (0)

template <typename T>
static cudaError_t galloc(T **p, size_t count)
{
    return cudaMalloc(reinterpret_cast<void **>(p), sizeof(T) * std::max<size_t>(count, 1));
}

template <typename T>
static void gfree(T *&p)
{
    if (p) cudaFree(p);
    p = nullptr;
}

// One matrix prepared for the network: the scaled matrix Ahat = -A / delta
// (delta = mean of diag(-A)) as its diagonal plus its off-diagonal part, its
// strict lower pattern and that pattern's transpose, the node features, and
// the work space of a pass.
struct cgb_gnn_graph {
    int n = 0;
    long long nnz_off = 0, nnz_low = 0;
    std::vector<double> dscale;   // 1/sqrt(delta) per row (host, FP64): F = G diag(dscale)
    int *off_ptr = nullptr, *off_col = nullptr;
    float *off_val = nullptr;
    float *adiag = nullptr;       // diagonal of Ahat
    int *low_ptr = nullptr, *low_col = nullptr;
    float *low_val = nullptr;
    int *up_ptr = nullptr, *up_row = nullptr, *up_map = nullptr;
    float *X = nullptr;
    std::vector<int> h_low_ptr, h_low_col;  // host copy of the strict lower pattern
    // forward cache
    float *Hs[kL + 1] = {nullptr, nullptr, nullptr, nullptr};
    float *T = nullptr, *U = nullptr;
    float *goff = nullptr, *gdiag = nullptr, *ud = nullptr;
    // training work space
    float *R = nullptr, *Pv = nullptr, *Q = nullptr, *Tg = nullptr, *Ug = nullptr, *W = nullptr;
    float *GU = nullptr, *GT = nullptr;
    float *dGoff = nullptr, *dGdiag = nullptr, *dv = nullptr;
    float *dh = nullptr, *dz = nullptr, *dT = nullptr;
};

struct cgb_gnn {
    int device = 0;
    int sms = 148;
    cudaStream_t stream = nullptr;
    float *P = nullptr, *G = nullptr, *M = nullptr, *V = nullptr;  // params, grad, Adam moments
    float *part = nullptr;   // kRedBlocks x 33 x 32
    float *colv = nullptr;   // small per-column vectors (8 x 32)
    float *loss = nullptr;
    int adam_t = 0;
};

namespace {

int grid_rows(const cgb_gnn *m, int n) { return std::max(1, std::min(8 * m->sms, (n + 7) / 8)); }

void free_graph(cgb_gnn_graph *g)
{
    if (!g) return;
    gfree(g->off_ptr); gfree(g->off_col); gfree(g->off_val);
    gfree(g->low_ptr); gfree(g->low_col); gfree(g->low_val);
    gfree(g->up_ptr); gfree(g->up_row); gfree(g->up_map);
    gfree(g->X); gfree(g->adiag);
    for (auto &h : g->Hs) gfree(h);
    gfree(g->T); gfree(g->U); gfree(g->goff); gfree(g->gdiag); gfree(g->ud);
    gfree(g->R); gfree(g->Pv); gfree(g->Q); gfree(g->Tg); gfree(g->Ug); gfree(g->W);
    gfree(g->GU); gfree(g->GT); gfree(g->dGoff); gfree(g->dGdiag); gfree(g->dv);
    gfree(g->dh); gfree(g->dz); gfree(g->dT);
    delete g;
}

// Deterministic initial weights: uniform(-a, a) from a hash of (seed, index),
// a = 1/sqrt(fan_in); head biases chosen so G starts near I - L (L the
// strict lower part of Ahat), whose G^T G ~ I - (Ahat - I) is the
// first-order inverse of Ahat: g_ii = 1, g_ij = -ahat_ij.
void init_params(std::vector<float> &p, unsigned seed)
{
    p.assign(kNumParams, 0.f);
    auto unif = [&](int idx, float a) {
        unsigned x = unsigned(idx) * 2654435761u + seed * 40503u + 12345u;
        x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
        return a * (2.f * (float(x >> 8) / 16777216.f) - 1.f);
    };
    for (int t = 0; t < kF * kH; t++) p[kOffWin + t] = unif(kOffWin + t, 1.f / std::sqrt(float(kF)));
    for (int l = 0; l < kL; l++) {
        const int o = kOffLayer + l * kLayerSize;
        for (int t = 0; t < 2 * kH * kH; t++) p[o + t] = unif(o + t, 1.f / std::sqrt(float(kH)));
    }
    for (int t = 0; t < kH; t++) {
        p[kOffWd + t] = 0.1f * unif(kOffWd + t, 1.f);
        p[kOffWe + t] = 0.1f * unif(kOffWe + t, 1.f);
    }
    p[kOffCd] = 0.5413249f;  // softplus^-1(1)
    p[kOffCe] = -1.0f;
}

// Forward pass on graph g: Hs[0..3], then G (goff, gdiag).
int forward(cgb_gnn *m, cgb_gnn_graph *g)
{
    const int n = g->n, gr = grid_rows(m, n);
    const float *P = m->P;
    k_dense<<<gr, 256, 0, m->stream>>>(g->X, kF, P + kOffWin, P + kOffBin, nullptr, g->Hs[0], n, 1);
    for (int l = 0; l < kL; l++) {
        const float *Ws = P + kOffLayer + l * kLayerSize;
        const float *Wm = Ws + kH * kH;
        const float *b = Wm + kH * kH;
        k_dense<<<gr, 256, 0, m->stream>>>(g->Hs[l], kH, Wm, nullptr, nullptr, g->T, n, 0);
        k_spmm<<<gr, 256, 0, m->stream>>>(g->off_ptr, g->off_col, g->off_val, nullptr, nullptr, 0.f,
                                         g->T, g->U, n);
        k_dense<<<gr, 256, 0, m->stream>>>(g->Hs[l], kH, Ws, b, g->U, g->Hs[l + 1], n, 1);
    }
    k_head<<<gr, 256, 0, m->stream>>>(g->Hs[kL], g->low_ptr, g->low_col, g->low_val, P, g->goff,
                                     g->gdiag, g->ud, n);
    GNN_TRY(cudaGetLastError());
    return CGB_OK;
}

// Y = Ahat X = diag(Ahat) X + Aoff X.
void ahat_mm(cgb_gnn *m, cgb_gnn_graph *g, const float *X, float *Y)
{
    k_spmm<<<grid_rows(m, g->n), 256, 0, m->stream>>>(g->off_ptr, g->off_col, g->off_val, nullptr,
                                                     g->adiag, 0.f, X, Y, g->n);
}
// Y = G X (lower pattern + diagonal)
void g_mm(cgb_gnn *m, cgb_gnn_graph *g, const float *X, float *Y)
{
    k_spmm<<<grid_rows(m, g->n), 256, 0, m->stream>>>(g->low_ptr, g->low_col, g->goff, nullptr,
                                                     g->gdiag, 0.f, X, Y, g->n);
}
// Y = G^T X (transposed pattern, values through the map)
void gt_mm(cgb_gnn *m, cgb_gnn_graph *g, const float *X, float *Y)
{
    k_spmm<<<grid_rows(m, g->n), 256, 0, m->stream>>>(g->up_ptr, g->up_row, g->goff, g->up_map,
                                                     g->gdiag, 0.f, X, Y, g->n);
}

// Column sums of a*b (b null: a*a) into m->colv + 32*slot.
void colsum(cgb_gnn *m, const float *a, const float *b, int n, int slot)
{
    k_colsum_prod<<<kRedBlocks, 256, 0, m->stream>>>(a, b, n, m->part);
    k_reduce_parts<<<1, 32, 0, m->stream>>>(m->part, kRedBlocks, kH, kH, m->colv + kH * slot, 0);
}

// Probes: 32 columns of R.  `cg_steps` = 0: normal random vectors; else the
// residuals after cg_steps batched CG steps on Ahat (from z0 = 0) for 32
// random right-hand sides.
int make_probes(cgb_gnn *m, cgb_gnn_graph *g, unsigned seed, int cg_steps)
{
    const int n = g->n;
    const size_t total = size_t(n) * kH;
    k_normal<<<grid_rows(m, n), 256, 0, m->stream>>>(g->R, total, seed);
    if (cg_steps > 0) {
        // R = b (random), r0 = b (z0 = 0), p0 = r0
        GNN_TRY(cudaMemcpyAsync(g->Pv, g->R, total * sizeof(float), cudaMemcpyDeviceToDevice, m->stream));
        float *rho = m->colv + 0 * kH, *pq = m->colv + 1 * kH, *alpha = m->colv + 2 * kH;
        float *rho_new = m->colv + 3 * kH, *beta = m->colv + 4 * kH;
        colsum(m, g->R, nullptr, n, 0);  // rho
        for (int s = 0; s < cg_steps; s++) {
            ahat_mm(m, g, g->Pv, g->Q);
            colsum(m, g->Pv, g->Q, n, 1);
            k_ratio<<<1, 32, 0, m->stream>>>(rho, pq, alpha);
            k_cg_update<<<grid_rows(m, n), 256, 0, m->stream>>>(g->R, g->Q, alpha, n);
            colsum(m, g->R, nullptr, n, 3);
            k_ratio<<<1, 32, 0, m->stream>>>(rho_new, rho, beta);
            k_cg_dir<<<grid_rows(m, n), 256, 0, m->stream>>>(g->Pv, g->R, beta, n);
            GNN_TRY(cudaMemcpyAsync(rho, rho_new, kH * sizeof(float), cudaMemcpyDeviceToDevice, m->stream));
        }
    }
    GNN_TRY(cudaGetLastError());
    return CGB_OK;
}

// Loss and gradient for the probes in g->R: fills m->G (all parameters)
// and *m->loss.
int loss_grad(cgb_gnn *m, cgb_gnn_graph *g)
{
    const int n = g->n, gr = grid_rows(m, n);
    const size_t total = size_t(n) * kH;
    int st = forward(m, g);
    if (st) return st;
    float *rn2 = m->colv + 5 * kH, *wn2 = m->colv + 6 * kH, *coef = m->colv + 7 * kH;
    colsum(m, g->R, nullptr, n, 5);
    g_mm(m, g, g->R, g->Tg);           // T = G R
    gt_mm(m, g, g->Tg, g->Ug);         // U = G^T T
    ahat_mm(m, g, g->Ug, g->W);        // W = Ahat U
    k_axpy_cols<<<gr, 256, 0, m->stream>>>(g->W, g->R, nullptr, g->W, n);  // W -= R
    colsum(m, g->W, nullptr, n, 6);
    k_loss_coef<<<1, 32, 0, m->stream>>>(rn2, wn2, coef, m->loss);
    ahat_mm(m, g, g->W, g->GU);        // GU = Ahat W, scaled per column
    k_axpy_cols<<<gr, 256, 0, m->stream>>>(g->GU, nullptr, coef, g->GU, n);
    g_mm(m, g, g->GU, g->GT);          // GT = G GU
    k_dG<<<gr, 256, 0, m->stream>>>(g->Tg, g->GU, g->GT, g->R, g->low_ptr, g->low_col, g->dGoff,
                                   g->dGdiag, n);
    // head backward
    k_head_bwd_rows<<<kRedBlocks, 256, 0, m->stream>>>(g->Hs[kL], g->low_ptr, g->low_col,
                                                      g->low_val, m->P, g->dGoff, g->dGdiag, g->ud,
                                                      g->dv, g->dh, m->part, n);
    k_reduce_parts<<<1, 96, 0, m->stream>>>(m->part, kRedBlocks, 66, 32, m->G + kOffWe, 0);
    k_reduce_parts<<<1, 96, 0, m->stream>>>(m->part + 32, kRedBlocks, 66, 32, m->G + kOffWd, 0);
    k_reduce_parts<<<1, 32, 0, m->stream>>>(m->part + 64, kRedBlocks, 66, 1, m->G + kOffCe, 0);
    k_reduce_parts<<<1, 32, 0, m->stream>>>(m->part + 65, kRedBlocks, 66, 1, m->G + kOffCd, 0);
    k_head_bwd_cols<<<gr, 256, 0, m->stream>>>(g->Hs[kL], g->up_ptr, g->up_row, g->up_map, m->P,
                                              g->dv, g->dh, n);
    // message-passing layers, last to first
    const int ostride = (kH + 1) * kH;
    for (int l = kL - 1; l >= 0; l--) {
        const float *Ws = m->P + kOffLayer + l * kLayerSize;
        const float *Wm = Ws + kH * kH;
        float *gWs = m->G + kOffLayer + l * kLayerSize;
        float *gWm = gWs + kH * kH;
        float *gb = gWm + kH * kH;
        k_relu_bwd<<<gr, 256, 0, m->stream>>>(g->dh, g->Hs[l + 1], g->dz, total);
        k_outer<<<kRedBlocks, 256, 0, m->stream>>>(g->Hs[l], kH, g->dz, n, m->part);
        k_reduce_parts<<<8, 128, 0, m->stream>>>(m->part, kRedBlocks, ostride, kH * kH, gWs, 0);
        k_reduce_parts<<<1, 32, 0, m->stream>>>(m->part + kH * kH, kRedBlocks, ostride, kH, gb, 0);
        k_spmm<<<gr, 256, 0, m->stream>>>(g->off_ptr, g->off_col, g->off_val, nullptr, nullptr, 0.f,
                                         g->dz, g->dT, n);  // dT = Aoff dz
        k_outer<<<kRedBlocks, 256, 0, m->stream>>>(g->Hs[l], kH, g->dT, n, m->part);
        k_reduce_parts<<<8, 128, 0, m->stream>>>(m->part, kRedBlocks, ostride, kH * kH, gWm, 0);
        k_dense_t2<<<gr, 256, 0, m->stream>>>(g->dz, Ws, g->dT, Wm, g->dh, n);
    }
    k_relu_bwd<<<gr, 256, 0, m->stream>>>(g->dh, g->Hs[0], g->dz, total);
    k_outer<<<kRedBlocks, 256, 0, m->stream>>>(g->X, kF, g->dz, n, m->part);
    k_reduce_parts<<<1, 128, 0, m->stream>>>(m->part, kRedBlocks, ostride, kF * kH, m->G + kOffWin, 0);
    k_reduce_parts<<<1, 32, 0, m->stream>>>(m->part + kH * kH, kRedBlocks, ostride, kH,
                                           m->G + kOffBin, 0);
    GNN_TRY(cudaGetLastError());
    return CGB_OK;
}

}  // namespace

extern "C" {

int cgb_gnn_param_count(void) { return kNumParams; }

int cgb_gnn_create(int device, unsigned seed, cgb_gnn **out)
{
    if (!out) return set_error(CGB_ERR_INVALID, "out is null");
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count)
        return set_error(CGB_ERR_NO_DEVICE, "no CUDA device %d", device);
    cudaDeviceProp prop;
    GNN_TRY(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) return set_error(CGB_ERR_NO_DEVICE, "device %d is not sm_100", device);
    GNN_TRY(cudaSetDevice(device));
    cgb_gnn *m = new (std::nothrow) cgb_gnn;
    if (!m) return set_error(CGB_ERR_NOMEM, "model allocation failed");
    m->device = device;
    m->sms = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess ||
        galloc(&m->P, kNumParams) || galloc(&m->G, kNumParams) || galloc(&m->M, kNumParams) ||
        galloc(&m->V, kNumParams) || galloc(&m->part, size_t(kRedBlocks) * (kH + 1) * kH) ||
        galloc(&m->colv, 8 * kH) || galloc(&m->loss, 1)) {
        cgb_gnn_destroy(m);
        return set_error(CGB_ERR_NOMEM, "model device allocation failed");
    }
    std::vector<float> p;
    init_params(p, seed);
    GNN_TRY(cudaMemcpy(m->P, p.data(), sizeof(float) * kNumParams, cudaMemcpyHostToDevice));
    GNN_TRY(cudaMemset(m->M, 0, sizeof(float) * kNumParams));
    GNN_TRY(cudaMemset(m->V, 0, sizeof(float) * kNumParams));
    *out = m;
    return CGB_OK;
}

int cgb_gnn_destroy(cgb_gnn *m)
{
    if (!m) return CGB_OK;
    cudaSetDevice(m->device);
    gfree(m->P); gfree(m->G); gfree(m->M); gfree(m->V); gfree(m->part); gfree(m->colv);
    gfree(m->loss);
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
    return CGB_OK;
}

int cgb_gnn_get_params(cgb_gnn *m, float *out, int count)
{
    if (!m || !out || count != kNumParams) return set_error(CGB_ERR_INVALID, "bad arguments");
    GNN_TRY(cudaSetDevice(m->device));
    GNN_TRY(cudaStreamSynchronize(m->stream));
    GNN_TRY(cudaMemcpy(out, m->P, sizeof(float) * kNumParams, cudaMemcpyDeviceToHost));
    return CGB_OK;
}

int cgb_gnn_set_params(cgb_gnn *m, const float *in, int count)
{
    if (!m || !in || count != kNumParams) return set_error(CGB_ERR_INVALID, "bad arguments");
    GNN_TRY(cudaSetDevice(m->device));
    GNN_TRY(cudaStreamSynchronize(m->stream));
    GNN_TRY(cudaMemcpy(m->P, in, sizeof(float) * kNumParams, cudaMemcpyHostToDevice));
    GNN_TRY(cudaMemset(m->M, 0, sizeof(float) * kNumParams));
    GNN_TRY(cudaMemset(m->V, 0, sizeof(float) * kNumParams));
    m->adam_t = 0;
    return CGB_OK;
}

int cgb_gnn_graph_create(cgb_gnn *m, int n, const int *rowstr, const int *colidx, const double *a,
                         cgb_gnn_graph **out)
{
    if (!m || !out || n < 2 || !rowstr || !colidx || !a)
        return set_error(CGB_ERR_INVALID, "bad arguments");
    *out = nullptr;
    GNN_TRY(cudaSetDevice(m->device));
    // host: D = diag(-A), scaled off-diagonal, strict lower pattern and its transpose
    std::vector<double> d(n, 0.0);
    for (int i = 0; i < n; i++)
        for (int k = rowstr[i]; k < rowstr[i + 1]; k++)
            if (colidx[k] == i) d[i] = -a[k];
    for (int i = 0; i < n; i++)
        if (!(d[i] > 0.0))
            return set_error(CGB_ERR_NUMERIC, "graph: diag(-A) not positive at row %d", i);
    cgb_gnn_graph *g = new (std::nothrow) cgb_gnn_graph;
    if (!g) return set_error(CGB_ERR_NOMEM, "graph allocation failed");
    g->n = n;
    double delta = 0.0;
    for (int i = 0; i < n; i++) delta += d[i];
    delta /= n;
    g->dscale.assign(n, 1.0 / std::sqrt(delta));
    std::vector<float> adiag(n);
    for (int i = 0; i < n; i++) adiag[i] = float(d[i] / delta);
    std::vector<int> optr(n + 1, 0), lptr(n + 1, 0), uptr(n + 1, 0);
    for (int i = 0; i < n; i++)
        for (int k = rowstr[i]; k < rowstr[i + 1]; k++) {
            const int j = colidx[k];
            if (j == i) continue;
            optr[i + 1]++;
            if (j < i) {
                lptr[i + 1]++;
                uptr[j + 1]++;
            }
        }
    for (int i = 0; i < n; i++) {
        optr[i + 1] += optr[i];
        lptr[i + 1] += lptr[i];
        uptr[i + 1] += uptr[i];
    }
    g->nnz_off = optr[n];
    g->nnz_low = lptr[n];
    std::vector<int> ocol(g->nnz_off), lcol(g->nnz_low), urow(g->nnz_low), umap(g->nnz_low);
    std::vector<float> oval(g->nnz_off), lval(g->nnz_low);
    std::vector<int> ucur(uptr.begin(), uptr.end() - 1);
    std::vector<float> X(size_t(n) * kF);
    double deg_sum = 0.0;
    for (int i = 0; i < n; i++) {
        int o = optr[i], l = lptr[i];
        float s = 0.f, t = 0.f;
        for (int k = rowstr[i]; k < rowstr[i + 1]; k++) {
            const int j = colidx[k];
            if (j == i) continue;
            const float v = float(-a[k] / delta);
            ocol[o] = j;
            oval[o++] = v;
            s += std::fabs(v);
            t += v;
            if (j < i) {
                lcol[l] = j;
                lval[l] = v;
                urow[ucur[j]] = i;
                umap[ucur[j]++] = l;
                l++;
            }
        }
        X[size_t(i) * kF + 0] = adiag[i];
        X[size_t(i) * kF + 1] = s;
        X[size_t(i) * kF + 2] = t;
        X[size_t(i) * kF + 3] = float(optr[i + 1] - optr[i]);
        deg_sum += optr[i + 1] - optr[i];
    }
    const float mean_deg = float(std::max(1.0, deg_sum / n));
    for (int i = 0; i < n; i++) X[size_t(i) * kF + 3] /= mean_deg;
    g->h_low_ptr = lptr;
    g->h_low_col = lcol;
    // the transposed pattern lists rows i in ascending order for each j
    const size_t nh = size_t(n) * kH;
    bool ok = !galloc(&g->off_ptr, n + 1) && !galloc(&g->off_col, g->nnz_off) &&
              !galloc(&g->off_val, g->nnz_off) && !galloc(&g->low_ptr, n + 1) &&
              !galloc(&g->low_col, g->nnz_low) && !galloc(&g->low_val, g->nnz_low) &&
              !galloc(&g->up_ptr, n + 1) && !galloc(&g->up_row, g->nnz_low) &&
              !galloc(&g->up_map, g->nnz_low) && !galloc(&g->X, size_t(n) * kF) &&
              !galloc(&g->T, nh) && !galloc(&g->U, nh) && !galloc(&g->goff, g->nnz_low) &&
              !galloc(&g->gdiag, n) && !galloc(&g->ud, n) && !galloc(&g->adiag, n);
    for (auto &h : g->Hs) ok = ok && !galloc(&h, nh);
    if (!ok) {
        free_graph(g);
        return set_error(CGB_ERR_NOMEM, "graph device allocation failed");
    }
    cudaMemcpy(g->off_ptr, optr.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice);
    cudaMemcpy(g->off_col, ocol.data(), sizeof(int) * g->nnz_off, cudaMemcpyHostToDevice);
    cudaMemcpy(g->off_val, oval.data(), sizeof(float) * g->nnz_off, cudaMemcpyHostToDevice);
    cudaMemcpy(g->low_ptr, lptr.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice);
    cudaMemcpy(g->low_col, lcol.data(), sizeof(int) * g->nnz_low, cudaMemcpyHostToDevice);
    cudaMemcpy(g->low_val, lval.data(), sizeof(float) * g->nnz_low, cudaMemcpyHostToDevice);
    cudaMemcpy(g->up_ptr, uptr.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice);
    cudaMemcpy(g->up_row, urow.data(), sizeof(int) * g->nnz_low, cudaMemcpyHostToDevice);
    cudaMemcpy(g->up_map, umap.data(), sizeof(int) * g->nnz_low, cudaMemcpyHostToDevice);
    cudaMemcpy(g->adiag, adiag.data(), sizeof(float) * n, cudaMemcpyHostToDevice);
    cudaError_t e = cudaMemcpy(g->X, X.data(), sizeof(float) * X.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        free_graph(g);
        return set_error(CGB_ERR_CUDA, "graph upload failed: %s", cudaGetErrorString(e));
    }
    *out = g;
    return CGB_OK;
}

int cgb_gnn_graph_destroy(cgb_gnn_graph *g)
{
    free_graph(g);
    return CGB_OK;
}

static int ensure_train_space(cgb_gnn_graph *g)
{
    if (g->R) return CGB_OK;
    const size_t nh = size_t(g->n) * kH;
    bool ok = !galloc(&g->R, nh) && !galloc(&g->Pv, nh) && !galloc(&g->Q, nh) &&
              !galloc(&g->Tg, nh) && !galloc(&g->Ug, nh) && !galloc(&g->W, nh) &&
              !galloc(&g->GU, nh) && !galloc(&g->GT, nh) && !galloc(&g->dGoff, g->nnz_low) &&
              !galloc(&g->dGdiag, g->n) && !galloc(&g->dv, g->nnz_low) && !galloc(&g->dh, nh) &&
              !galloc(&g->dz, nh) && !galloc(&g->dT, nh);
    return ok ? CGB_OK : set_error(CGB_ERR_NOMEM, "training work space allocation failed");
}

int cgb_gnn_loss_grad(cgb_gnn *m, cgb_gnn_graph *g, const float *probes, unsigned seed,
                      int cg_steps, float *loss, float *grad)
{
    if (!m || !g || cg_steps < 0 || cg_steps > 64) return set_error(CGB_ERR_INVALID, "bad arguments");
    GNN_TRY(cudaSetDevice(m->device));
    int st = ensure_train_space(g);
    if (st) return st;
    if (probes) {
        GNN_TRY(cudaMemcpyAsync(g->R, probes, sizeof(float) * size_t(g->n) * kH,
                                cudaMemcpyHostToDevice, m->stream));
    } else {
        st = make_probes(m, g, seed, cg_steps);
        if (st) return st;
    }
    st = loss_grad(m, g);
    if (st) return st;
    GNN_TRY(cudaStreamSynchronize(m->stream));
    if (loss) GNN_TRY(cudaMemcpy(loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost));
    if (grad) GNN_TRY(cudaMemcpy(grad, m->G, sizeof(float) * kNumParams, cudaMemcpyDeviceToHost));
    return CGB_OK;
}

int cgb_gnn_train_step(cgb_gnn *m, cgb_gnn_graph *g, unsigned seed, int cg_steps, float lr,
                       float *loss)
{
    if (!m || !g || !(lr > 0.f) || cg_steps < 0 || cg_steps > 64)
        return set_error(CGB_ERR_INVALID, "bad arguments");
    GNN_TRY(cudaSetDevice(m->device));
    int st = ensure_train_space(g);
    if (st) return st;
    st = make_probes(m, g, seed, cg_steps);
    if (st) return st;
    st = loss_grad(m, g);
    if (st) return st;
    m->adam_t++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, float(m->adam_t)), c2 = 1.f - std::pow(b2, float(m->adam_t));
    k_adam<<<(kNumParams + 255) / 256, 256, 0, m->stream>>>(m->P, m->G, m->M, m->V, kNumParams, lr,
                                                           b1, b2, 1e-8f, c1, c2);
    GNN_TRY(cudaGetLastError());
    if (loss) {
        GNN_TRY(cudaMemcpyAsync(loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    }
    GNN_TRY(cudaStreamSynchronize(m->stream));
    return CGB_OK;
}

// Inference: G for graph g.  goff (nnz_low, the strict lower pattern in row
// order) and gdiag (n) are device or host pointers (host when to_host).
int cgb_gnn_infer(cgb_gnn *m, cgb_gnn_graph *g, float *goff_host, float *gdiag_host)
{
    if (!m || !g) return set_error(CGB_ERR_INVALID, "bad arguments");
    GNN_TRY(cudaSetDevice(m->device));
    int st = forward(m, g);
    if (st) return st;
    GNN_TRY(cudaStreamSynchronize(m->stream));
    if (goff_host)
        GNN_TRY(cudaMemcpy(goff_host, g->goff, sizeof(float) * g->nnz_low, cudaMemcpyDeviceToHost));
    if (gdiag_host)
        GNN_TRY(cudaMemcpy(gdiag_host, g->gdiag, sizeof(float) * g->n, cudaMemcpyDeviceToHost));
    return CGB_OK;
}

// F = G / sqrt(delta) on the lower pattern of A (strictly lower entries in
// column order, then the diagonal) as CSR.
static int learned_factor(cgb_gnn *m, cgb_gnn_graph *g, std::vector<int> &fptr,
                          std::vector<int> &fcol, std::vector<double> &fval)
{
    const int n = g->n;
    std::vector<float> goff(g->nnz_low), gdiag(n);
    int st = cgb_gnn_infer(m, g, goff.data(), gdiag.data());
    if (st) return st;
    fptr.assign(n + 1, 0);
    fcol.assign(g->nnz_low + n, 0);
    fval.assign(g->nnz_low + n, 0.0);
    long long at = 0;
    for (int i = 0; i < n; i++) {
        fptr[i] = int(at);
        for (int k = g->h_low_ptr[i]; k < g->h_low_ptr[i + 1]; k++) {
            const int j = g->h_low_col[k];
            fcol[at] = j;
            fval[at++] = double(goff[k]) * g->dscale[j];
        }
        fcol[at] = i;
        fval[at++] = double(gdiag[i]) * g->dscale[i];
    }
    fptr[n] = int(at);
    return CGB_OK;
}

// The learned factor as system `sys`'s preconditioner in a batch.
int cgb_gnn_attach_batch(cgb_gnn *m, cgb_gnn_graph *g, cgb_batch *b, int sys)
{
    if (!m || !g || !b) return set_error(CGB_ERR_INVALID, "bad arguments");
    std::vector<int> fptr, fcol;
    std::vector<double> fval;
    int st = learned_factor(m, g, fptr, fcol, fval);
    if (st) return st;
    return cgb_batch_set_preconditioner(b, sys, fptr.data(), fcol.data(), fval.data());
}

// Learned preconditioner into a session: F = G / sqrt(delta) on the lower
// pattern of A (strictly lower entries in column order, then the diagonal).
int cgb_gnn_attach(cgb_gnn *m, cgb_gnn_graph *g, cgb_session *s)
{
    if (!m || !g || !s) return set_error(CGB_ERR_INVALID, "bad arguments");
    const int n = g->n;
    std::vector<float> goff(g->nnz_low), gdiag(n);
    int st = cgb_gnn_infer(m, g, goff.data(), gdiag.data());
    if (st) return st;
    std::vector<int> fptr(n + 1, 0), fcol(g->nnz_low + n);
    std::vector<double> fval(g->nnz_low + n);
    long long at = 0;
    for (int i = 0; i < n; i++) {
        fptr[i] = int(at);
        for (int k = g->h_low_ptr[i]; k < g->h_low_ptr[i + 1]; k++) {
            const int j = g->h_low_col[k];
            fcol[at] = j;
            fval[at++] = double(goff[k]) * g->dscale[j];
        }
        fcol[at] = i;
        fval[at++] = double(gdiag[i]) * g->dscale[i];
    }
    fptr[n] = int(at);
    return cgb_set_preconditioner(s, fptr.data(), fcol.data(), fval.data());
}

int cgb_gnn_graph_info(cgb_gnn_graph *g, int *n, long long *nnz_low, double *dscale_out)
{
    if (!g) return set_error(CGB_ERR_INVALID, "graph is null");
    if (n) *n = g->n;
    if (nnz_low) *nnz_low = g->nnz_low;
    if (dscale_out) std::memcpy(dscale_out, g->dscale.data(), sizeof(double) * g->n);
    return CGB_OK;
}

}  // extern "C"
