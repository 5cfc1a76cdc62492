// queries.cu - ray queries used for parity checks: closest hit of arbitrary
// rays and of camera rays (Camera::ray_at then Scene::hit).
#include <cuda_runtime.h>

#include "host_internal.h"
#include "path.cuh"

namespace pgpu {

constexpr int kQShared = 16;

template <bool CAMERA>
__global__ void __launch_bounds__(128)
query_closest(SceneView S, const float* __restrict__ in, int n, int* __restrict__ prim_out,
              float* __restrict__ t_out) {
    extern __shared__ int smem[];
    TravStack<kQShared> stk;
    stk.sref = smem + threadIdx.x;
    stk.st = reinterpret_cast<float*>(smem + kQShared * blockDim.x) + threadIdx.x;
    stk.stride = blockDim.x;
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    Ray r;
    if (CAMERA) {
        r = camera_ray(S.cam, in[2 * k], in[2 * k + 1]);
    } else {
        r.o = v3(in[6 * k], in[6 * k + 1], in[6 * k + 2]);
        r.d = v3(in[6 * k + 3], in[6 * k + 4], in[6 * k + 5]);
    }
    float tb;
    int bref;
    int slot = closest_hit<kQShared, false>(S, r, 1e-4f, 1e9f, tb, bref, stk, nullptr);
    prim_out[k] = slot >= 0 ? __ldg(S.leaf_prim + slot) : -1;
    t_out[k] = slot >= 0 ? tb : -1.0f;
}

cudaError_t launch_query(const SceneView& S, bool camera, const float* in, int n, int* prim,
                         float* t, cudaStream_t st) {
    const int block = 128;
    int blocks = (n + block - 1) / block;
    size_t smem = (size_t)kQShared * block * 8;
    if (n <= 0) return cudaSuccess;
    if (camera) query_closest<true><<<blocks, block, smem, st>>>(S, in, n, prim, t);
    else query_closest<false><<<blocks, block, smem, st>>>(S, in, n, prim, t);
    return cudaGetLastError();
}

}  // namespace pgpu
