// pb_mlp_host.cuh - host side of the learned scheduler's network: parameter
// layout, initialisation, training loop (Adam) and inference.
//
// Flat FP32 parameter layout (also the layout of pb_mlp_get/set_params):
//   [ W1 781x256 | b1 256 | W2 256x256 | b2 256 | W3 256x4 | b3 4 ]
// W1 rows are input features, W2[i][j] maps hidden-1 unit i to hidden-2
// unit j, W3[j][o] maps hidden-2 unit j to output o.
#pragma once
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "pb_mlp.cuh"
#include "pb_util.cuh"

namespace pb {

constexpr size_t MLP_OFF_W1 = 0;
constexpr size_t MLP_OFF_B1 = MLP_OFF_W1 + (size_t)MLP_IN * MLP_H;
constexpr size_t MLP_OFF_W2 = MLP_OFF_B1 + MLP_H;
constexpr size_t MLP_OFF_B2 = MLP_OFF_W2 + (size_t)MLP_H * MLP_H;
constexpr size_t MLP_OFF_W3 = MLP_OFF_B2 + MLP_H;
constexpr size_t MLP_OFF_B3 = MLP_OFF_W3 + (size_t)MLP_H * MLP_OUT;
constexpr size_t MLP_PARAMS = MLP_OFF_B3 + MLP_OUT;

// An owning device array, freed when it leaves scope.
template <class T>
struct DeviceBuffer {
    T *p = nullptr;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer &) = delete;
    DeviceBuffer &operator=(const DeviceBuffer &) = delete;
    ~DeviceBuffer()
    {
        if (p) cudaFree(p);
    }
    cudaError_t alloc(size_t n) { return cudaMalloc(reinterpret_cast<void **>(&p), n * sizeof(T)); }
};

struct Mlp {
    bool ready = false;
    int max_batch = 0;
    u64 step = 0;
    // parameters, gradients, Adam moments (FP32) and the BF16 copy
    float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
    __nv_bfloat16 *pb = nullptr;
    // activations for one batch
    int16_t *idx = nullptr;
    float *h1f = nullptr, *z2 = nullptr, *h2f = nullptr, *y = nullptr, *dy = nullptr, *dh2f = nullptr,
          *dh1 = nullptr, *t = nullptr, *loss = nullptr;
    u32 *err = nullptr;     // GEMM error word (a tensor-core wait that gave up)
    float *work = nullptr;  // GEMM K-split partial tiles
    static constexpr size_t WORK_ELEMS = (size_t)tc::MAX_SPLITS * MLP_H * MLP_H;
    __nv_bfloat16 *h1b = nullptr, *h2b = nullptr, *dh2b = nullptr;
    Board *pos_b = nullptr;
    uint8_t *pos_s = nullptr, *pos_c = nullptr;

    void release()
    {
        void *ptrs[] = {p,   g,   m,   v,   pb,  idx,  h1f,  z2,    h2f,   y,     dy,
                        dh2f, dh1, t, loss, err, work, h1b, h2b, dh2b, pos_b, pos_s, pos_c};
        for (void *q : ptrs)
            if (q) cudaFree(q);
        *this = Mlp();
    }

    cudaError_t alloc_batch(int B)
    {
        if (B <= max_batch) return cudaSuccess;
        void *old[] = {idx, h1f, z2, h2f, y, dy, dh2f, dh1, t, h1b, h2b, dh2b, pos_b, pos_s, pos_c};
        for (void *q : old)
            if (q) cudaFree(q);
        cudaError_t e;
        size_t H = (size_t)B * MLP_H;
#define PB_MLP_ALLOC(ptr, bytes) \
    if ((e = cudaMalloc(reinterpret_cast<void **>(&ptr), bytes)) != cudaSuccess) return e;
        PB_MLP_ALLOC(idx, (size_t)B * MLP_MAX_ACTIVE * sizeof(int16_t));
        PB_MLP_ALLOC(h1f, H * 4);
        PB_MLP_ALLOC(z2, H * 4);
        PB_MLP_ALLOC(h2f, H * 4);
        PB_MLP_ALLOC(dh2f, H * 4);
        PB_MLP_ALLOC(dh1, H * 4);
        PB_MLP_ALLOC(h1b, H * 2);
        PB_MLP_ALLOC(h2b, H * 2);
        PB_MLP_ALLOC(dh2b, H * 2);
        PB_MLP_ALLOC(y, (size_t)B * MLP_OUT * 4);
        PB_MLP_ALLOC(dy, (size_t)B * MLP_OUT * 4);
        PB_MLP_ALLOC(t, (size_t)B * MLP_OUT * 4);
        PB_MLP_ALLOC(pos_b, (size_t)B * sizeof(Board));
        PB_MLP_ALLOC(pos_s, (size_t)B);
        PB_MLP_ALLOC(pos_c, (size_t)B);
#undef PB_MLP_ALLOC
        max_batch = B;
        return cudaSuccess;
    }

    // He-uniform weights from a splitmix64 stream, zero biases (b3 = out_bias).
    cudaError_t init(u64 seed, const float *out_bias, cudaStream_t s)
    {
        release();
        cudaError_t e;
        size_t bytes = MLP_PARAMS * sizeof(float);
        if ((e = cudaMalloc(&p, bytes)) != cudaSuccess) return e;
        if ((e = cudaMalloc(&g, bytes)) != cudaSuccess) return e;
        if ((e = cudaMalloc(&m, bytes)) != cudaSuccess) return e;
        if ((e = cudaMalloc(&v, bytes)) != cudaSuccess) return e;
        if ((e = cudaMalloc(&pb, MLP_PARAMS * sizeof(__nv_bfloat16))) != cudaSuccess) return e;
        if ((e = cudaMalloc(&loss, 64)) != cudaSuccess) return e;
        if ((e = cudaMalloc(&err, sizeof(u32))) != cudaSuccess) return e;
        if ((e = cudaMalloc(&work, WORK_ELEMS * sizeof(float))) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(err, 0, sizeof(u32), s)) != cudaSuccess) return e;
        std::vector<float> h(MLP_PARAMS, 0.f);
        u64 st = seed;
        auto uni = [&](float lim) {
            u64 r = splitmix64(&st);
            return lim * (2.0f * (float)((r >> 11) * (1.0 / 9007199254740992.0)) - 1.0f);
        };
        // layer 1 sees ~35 active inputs of 781, so scale by the active fan-in
        float l1 = sqrtf(6.f / 35.f), l2 = sqrtf(6.f / MLP_H), l3 = sqrtf(3.f / MLP_H);
        for (size_t i = 0; i < (size_t)MLP_IN * MLP_H; i++) h[MLP_OFF_W1 + i] = uni(l1);
        for (size_t i = 0; i < (size_t)MLP_H * MLP_H; i++) h[MLP_OFF_W2 + i] = uni(l2);
        for (size_t i = 0; i < (size_t)MLP_H * MLP_OUT; i++) h[MLP_OFF_W3 + i] = uni(l3);
        if (out_bias)
            for (int o = 0; o < MLP_OUT; o++) h[MLP_OFF_B3 + o] = out_bias[o];
        if ((e = set_params(h.data(), s)) != cudaSuccess) return e;
        step = 0;
        ready = true;
        return cudaSuccess;
    }

    cudaError_t set_params(const float *host, cudaStream_t s)
    {
        cudaError_t e;
        size_t bytes = MLP_PARAMS * sizeof(float);
        if ((e = cudaMemcpyAsync(p, host, bytes, cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(m, 0, bytes, s)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(v, 0, bytes, s)) != cudaSuccess) return e;
        k_to_bf16<<<(unsigned)((MLP_PARAMS + 255) / 256), 256, 0, s>>>(p, MLP_PARAMS, pb);
        step = 0;
        return cudaGetLastError();
    }

    // Positions -> feature indices (device), for rows [0, n) of the batch buffers.
    cudaError_t load_positions(const pb_pos *pos, int n, cudaStream_t s) { return features_to(pos, n, idx, s); }

    // Feature indices of n positions (n <= max_batch) into rows [0, n) of `out`.
    cudaError_t features_to(const pb_pos *pos, int n, int16_t *out, cudaStream_t s)
    {
        std::vector<Board> b(n);
        std::vector<uint8_t> st(n), col(n);
        for (int i = 0; i < n; i++) {
            for (int k = 0; k < 4; k++) b[i].bb[k] = pos[i].bb[k];
            st[i] = pos[i].state;
            col[i] = pos[i].color;
        }
        cudaError_t e;
        if ((e = cudaMemcpyAsync(pos_b, b.data(), sizeof(Board) * n, cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
        if ((e = cudaMemcpyAsync(pos_s, st.data(), n, cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
        if ((e = cudaMemcpyAsync(pos_c, col.data(), n, cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
        k_features<<<(n + 255) / 256, 256, 0, s>>>(pos_b, pos_s, pos_c, n, out);
        return cudaGetLastError();
    }

    // Forward over rows [0, B) (B a multiple of 64); with targets also the
    // loss, its gradient and all parameter gradients.
    cudaError_t forward_backward(int B, bool with_grad, cudaStream_t s)
    {
        const __nv_bfloat16 *w1 = pb + MLP_OFF_W1, *w2 = pb + MLP_OFF_W2, *w3 = pb + MLP_OFF_W3;
        k_mlp_layer1<<<B, MLP_H, 0, s>>>(idx, w1, p + MLP_OFF_B1, B, h1f, h1b);
        cudaError_t e =
            gemm_tc<false, false>(h1b, MLP_H, w2, MLP_H, z2, MLP_H, B, MLP_H, MLP_H, err, work, WORK_ELEMS, s);
        if (e != cudaSuccess) return e;
        size_t H = (size_t)B * MLP_H;
        k_bias_relu<<<(unsigned)((H + 255) / 256), 256, 0, s>>>(z2, p + MLP_OFF_B2, B, h2f, h2b);
        if (with_grad) cudaMemsetAsync(loss, 0, sizeof(float), s);
        k_mlp_out<<<(B * 32 + 255) / 256, 256, 0, s>>>(h2f, w3, p + MLP_OFF_B3, B, y, with_grad ? t : nullptr, dy,
                                                       loss);
        if (!with_grad) return cudaGetLastError();
        k_grad_w3<<<MLP_H + 1, 256, 0, s>>>(h2f, dy, B, g + MLP_OFF_W3, g + MLP_OFF_B3);
        k_back_h2<<<(unsigned)((H + 255) / 256), 256, 0, s>>>(dy, w3, h2f, B, dh2f, dh2b);
        k_colsum<<<1, MLP_H, 0, s>>>(dh2f, B, g + MLP_OFF_B2);
        // dW2 = h1^T dh2 ; dh1 = dh2 W2^T
        if ((e = gemm_tc<true, false>(h1b, MLP_H, dh2b, MLP_H, g + MLP_OFF_W2, MLP_H, MLP_H, MLP_H, B, err, work,
                                      WORK_ELEMS, s)) != cudaSuccess)
            return e;
        if ((e = gemm_tc<false, true>(dh2b, MLP_H, w2, MLP_H, dh1, MLP_H, B, MLP_H, MLP_H, err, work, WORK_ELEMS,
                                      s)) != cudaSuccess)
            return e;
        cudaMemsetAsync(g + MLP_OFF_W1, 0, sizeof(float) * ((size_t)MLP_IN * MLP_H + MLP_H), s);
        k_back_l1<<<B, MLP_H, 0, s>>>(idx, dh1, h1f, B, g + MLP_OFF_W1, g + MLP_OFF_B1);
        return cudaGetLastError();
    }

    cudaError_t adam_step(float lr, cudaStream_t s)
    {
        const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
        step++;
        float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
        k_adam<<<(unsigned)((MLP_PARAMS + 255) / 256), 256, 0, s>>>(p, g, m, v, pb, MLP_PARAMS, lr, b1, b2, eps, c1,
                                                                    c2);
        return cudaGetLastError();
    }
};

}  // namespace pb
